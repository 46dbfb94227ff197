"""GPU parity against the CPU oracle, through the C ABI (libhh_cuda.so)."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import lib_params, lib_system, oracle_params, oracle_system, rel_to_c0

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from hawaiihybrid_b200 import _lib
    return _lib.load()


def test_mt_stream_bit_exact(lib):
    lib_system("hear")
    for seed in (42, 7, 1):
        n = 200_000
        out = np.empty(n, dtype=np.uint32)
        assert lib.hh_cuda_mt_stream(seed, n, out) == 0
        assert np.array_equal(out, O.mt_stream(seed, n))
    assert abs(out[:1].astype(np.float64)[0] * 2.0 ** -32 - O.mt_stream(1, 1)[0] * 2.0 ** -32) == 0


@pytest.mark.parametrize("n", [3_000_000, 45_000_000])
def test_mt_stream_segmented_bit_exact(lib, n):
    """Long requests are generated in segments from jumped-ahead states (fine jumps only
    for 3e6 words; coarse and fine jumps for 4.5e7): every word equals the sequential
    stream of the oracle."""
    lib_system("hear")
    out = np.empty(n, dtype=np.uint32)
    assert lib.hh_cuda_mt_stream(2066497031, n, out) == 0
    ref = O.mt_stream(2066497031, n)
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("name,seed,T,n", [("hear", 42, 300.0, 3000), ("co2ar", 7, 300.0, 3000),
                                           ("hear", 5, 100.0, 1000), ("co2ar", 11, 150.0, 1000)])
def test_sampler_matches_oracle(name, seed, T, n):
    import hawaiihybrid_b200 as hh
    ms = lib_system(name, seed)
    p = lib_params(name, 64, 100.0)
    qp, cand = hh.sample_initial_conditions(ms, p, T, n, seed=seed)
    qp_ref, cand_ref = O.sample(seed, oracle_system(name), oracle_params(name, 64, 100.0), T, n)
    assert cand == cand_ref
    # same candidates accepted in the same order; values agree to libm rounding
    np.testing.assert_allclose(qp, qp_ref, rtol=1e-13, atol=1e-300)


def test_sampler_stream_continues(lib):
    """seed == 0 continues the stream, as consecutive iterations of the reference do."""
    import hawaiihybrid_b200 as hh
    ms = lib_system("co2ar", 3)
    p = lib_params("co2ar", 64, 100.0)
    a, _ = hh.sample_initial_conditions(ms, p, 300.0, 500, seed=3)
    b, _ = hh.sample_initial_conditions(ms, p, 300.0, 700, seed=0)
    ref, _ = O.sample(3, oracle_system("co2ar"), oracle_params("co2ar", 64, 100.0), 300.0, 1200)
    np.testing.assert_allclose(np.vstack([a, b]), ref, rtol=1e-13, atol=1e-300)


@pytest.mark.parametrize("name,N,dt,n", [("hear", 2048, 200.0, 256), ("co2ar", 4096, 100.0, 128)])
def test_fp64_correlation_matches_oracle(name, N, dt, n):
    import hawaiihybrid_b200 as hh
    ms = lib_system(name)
    qp, _ = O.sample(42, oracle_system(name), oracle_params(name, N, dt), 300.0, n)
    crln, st = hh.correlation_from_initial_conditions(ms, lib_params(name, N, dt), qp)
    ref = O.correlation_sum(oracle_system(name), oracle_params(name, N, dt), qp)
    assert st.n_failed == 0
    # same integrator family at rtol 1e-12 in two coordinate systems
    assert rel_to_c0(crln, ref) < 1e-7


@pytest.mark.parametrize("name,dt", [("hear", 200.0), ("co2ar", 100.0)])
def test_single_trajectory_early_times(name, dt):
    """Per-trajectory C_i(t_k) over the first 1000 a.u. against the oracle, 1e-9 of C_i(0)."""
    import hawaiihybrid_b200 as hh
    ms = lib_system(name)
    qp, _ = O.sample(9, oracle_system(name), oracle_params(name, 64, dt), 300.0, 16)
    kmax = int(1000.0 / dt) + 1
    for i in range(qp.shape[0]):
        crln, _ = hh.correlation_from_initial_conditions(ms, lib_params(name, 64, dt), qp[i:i + 1])
        ref, st = O.correlation_eval(oracle_system(name), oracle_params(name, 64, dt), qp[i])
        assert np.max(np.abs(crln[:kmax] - ref[:kmax])) <= 1e-9 * abs(ref[0])


@pytest.mark.parametrize("name,N,dt,n,window", [("hear", 4096, 200.0, 2048, 4096),
                                                  ("co2ar", 4096, 100.0, 2048, 1001)])
def test_mixed_matches_fp64(name, N, dt, n, window):
    """The mixed path against the FP64 path on the same initial conditions: M0 (from C(0))
    and C(t) within 1e-4 of C(0).  He-Ar is compared over the whole window; for CO2-Ar the
    comparison covers t <= 1e5 a.u. (the collision window), because later samples are
    dominated by long-lived chaotic complexes whose pointwise C(t) is not reproducible even
    between two FP64 runs at rtol 1e-12 and 1e-13."""
    import hawaiihybrid_b200 as hh
    ms = lib_system(name)
    p = lib_params(name, N, dt)
    c64, _, s64 = hh.correlation_iteration(ms, p, 300.0, n, hh.PRECISION_FP64, seed=5)
    c32, _, s32 = hh.correlation_iteration(ms, p, 300.0, n, hh.PRECISION_MIXED, seed=5)
    assert rel_to_c0(c32[:window], c64[:window]) <= 1e-4
    assert abs(c32[0] - c64[0]) / abs(c64[0]) <= 1e-6   # M0 from C(0)


@pytest.mark.parametrize("name", ["hear", "co2ar"])
def test_m0_matches_oracle(name):
    import hawaiihybrid_b200 as hh
    ms = lib_system(name)
    p = lib_params(name, 64, 100.0)
    T = np.linspace(150.0, 400.0, 16)
    n = 400_000
    m64, e64 = hh.calculate_m0(ms, p, T, n, seed=99, precision=hh.PRECISION_FP64)
    m32, e32 = hh.calculate_m0(ms, p, T, n, seed=99, precision=hh.PRECISION_MIXED)
    ws, wq = O.m0(oracle_system(name), oracle_params(name, 64, 100.0), T, n, 99)
    mref = O.m0_scale(oracle_params(name, 64, 100.0)) * ws / n
    np.testing.assert_allclose(m64, mref, rtol=1e-10)
    np.testing.assert_allclose(m32, m64, rtol=1e-4)


def test_idct_golden():
    import os
    import hawaiihybrid_b200 as hh
    lib_system("hear")
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "cf_sf_he_ar_1000.npz"))
    N = g["cf"].size
    cf = hh.CFnc(t=g["dt"] * np.arange(N), data=g["cf"].copy(), ntraj=float(g["ntraj"]),
                 Temperature=float(g["temperature"]), normalized=True)
    sf = hh.idct_cf_to_sf(cf)
    peak = np.max(np.abs(g["sf"]))
    assert np.max(np.abs(sf.data - g["sf"])) / peak < 1e-6
    m = np.abs(g["sf"]) >= 1e-6 * peak
    assert np.max(np.abs(sf.data[m] - g["sf"][m]) / np.abs(g["sf"][m])) < 1e-6
    np.testing.assert_allclose(sf.nu[::64][1:], g["sf_nu_every64"][1:], rtol=1e-9)


def test_idct_graph_replay_and_recapture():
    """The CF->SF kernels run as a captured CUDA graph: repeated calls replay it, a new
    length or time step captures a new one; every result matches the oracle."""
    import hawaiihybrid_b200 as hh
    lib_system("hear")
    rng = np.random.default_rng(4)
    for N, dt in ((4096, 200.0), (4096, 200.0), (1024, 200.0), (4096, 100.0), (4096, 200.0)):
        data = np.exp(-np.arange(N) / (0.1 * N)) * (1 + 0.01 * rng.standard_normal(N))
        cf = hh.CFnc(t=dt * np.arange(N), data=data.copy(), ntraj=1.0, Temperature=300.0, normalized=True)
        sf = hh.idct_cf_to_sf(cf)
        nu_ref, sf_ref, cf_ref = O.idct_cf_to_sf(data, dt)
        peak = np.max(np.abs(sf_ref))
        assert np.max(np.abs(sf.data - sf_ref)) <= 1e-12 * peak
        np.testing.assert_allclose(sf.nu, nu_ref, rtol=1e-12)
        np.testing.assert_allclose(cf.data, cf_ref, rtol=0, atol=1e-15)


@pytest.mark.parametrize("status,hard", [(3, True), (5, True), (1, False)])
def test_failure_semantics(lib, status, hard):
    """A branch ending in a hard failure drops the whole trajectory (still counted);
    an integrator failure keeps the samples taken before it (src/hawaii.c:2172-2243, 3001)."""
    import hawaiihybrid_b200 as hh
    name, N, dt = "hear", 512, 200.0
    ms = lib_system(name)
    qp, _ = O.sample(21, oracle_system(name), oracle_params(name, N, dt), 300.0, 32)
    traj, k_fail = 5, 3
    assert lib.hh_cuda_debug_inject(traj, 0, k_fail, status) == 0
    try:
        crln, st = hh.correlation_from_initial_conditions(ms, lib_params(name, N, dt), qp)
    finally:
        lib.hh_cuda_debug_inject(-1, 0, 0, 0)
    keep = [i for i in range(qp.shape[0]) if i != traj]
    ref = O.correlation_sum(oracle_system(name), oracle_params(name, N, dt), qp[keep])
    if not hard:
        # forward branch of `traj` truncated before sample k_fail, backward branch intact
        full, _ = O.correlation_eval(oracle_system(name), oracle_params(name, N, dt), qp[traj])
        fw_bw = O.correlation_parts(oracle_system(name), oracle_params(name, N, dt), qp[traj])
        fw, bw = fw_bw
        fw[k_fail:] = 0.0
        ref = ref + 0.5 * (fw + bw) * (5.29177210903e-11) ** 3
    assert st.n_failed == (1 if hard else 0)
    assert rel_to_c0(crln, ref) < 1e-7


def test_multi_iteration_matches_consecutive_calls(lib):
    """Iterations in one launch equal consecutive single-iteration calls on the same stream."""
    import hawaiihybrid_b200 as hh
    ms = lib_system("co2ar", 13)
    p = lib_params("co2ar", 1024, 100.0)
    c_multi, nt, st = hh.correlation_iterations(ms, p, 300.0, 300, 3, hh.PRECISION_FP64, seed=13)
    singles = [hh.correlation_iteration(ms, p, 300.0, 300, hh.PRECISION_FP64, seed=(13 if i == 0 else 0))[0]
               for i in range(3)]
    for i in range(3):
        assert rel_to_c0(c_multi[i], singles[i]) < 1e-12
    assert list(nt) == [300.0, 300.0, 300.0]


@pytest.mark.parametrize("name", ["hear", "co2ar", "n2ar"])
def test_m2_matches_oracle(name):
    """M2 on the device (Cartesian central differences of the FP64 lab dipole) against
    the oracle's restatement in the reference's coordinates, on the same Philox samples:
    the two difference schemes agree to their truncation error."""
    import hawaiihybrid_b200 as hh
    ms = lib_system(name)
    p = lib_params(name, 64, 100.0)
    T = np.array([100.0, 200.0, 300.0])
    n = 1 << 16
    m, e = hh.calculate_m2(ms, p, T, n, seed=99)
    ws, wq = O.m2(oracle_system(name), oracle_params(name, 64, 100.0), T, n, 99)
    mref = O.m2_scale(oracle_params(name, 64, 100.0)) * ws / n
    np.testing.assert_allclose(m, mref, rtol=1e-5)
    assert np.all(e > 0) and np.all(e < 0.2 * m)


@pytest.mark.parametrize("name,T,Rmin,published", [
    ("co2ar", 100.0, 4.0, 4.41296e-01),   # example_configs/CF-F-CO2-Ar.conf.out:238 (VEGAS), +- 0.08 %
    ("hear", 100.0, 3.0, 1.34536e-02),    # example_configs/CF-F-He-Ar.conf.out:239 (VEGAS), +- 0.02 %
])
def test_m2_physics_anchor(name, T, Rmin, published):
    """M2 from 2^26 device samples against the reference's published VEGAS values:
    within 0.3 % plus three standard errors."""
    import hawaiihybrid_b200 as hh
    ms = lib_system(name)
    m, e = hh.calculate_m2(ms, lib_params(name, 64, 100.0, Rmin=Rmin), [T], 1 << 26, seed=7)
    assert abs(m[0] - published) <= 3e-3 * published + 3 * e[0]


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name,T,N,dt", [("hear", 300.0, 1024, 200.0), ("co2ar", 300.0, 1024, 100.0),
                                         ("ch4co2", 300.0, 64, 200.0)])
def test_solo_kernel_follows_the_bulk_path(name, T, N, dt, precision):
    """The solo kernel (one trajectory per warp, one state component per lane) takes over
    the last open items of a launch and runs launches with no more items than its warp
    slots.  Its stage sums, error norm and dense output keep the per-lane operations and
    their order, so every half-trajectory takes the same steps in either kernel: a
    2500-trajectory launch (bulk, then hand-off) against the same trajectories in five
    launches of 500 (solo only), per item, and the sum of their C(t) against its C(t)."""
    import hawaiihybrid_b200 as hh
    ms = lib_system(name)
    L = _lib_handle()
    p = lib_params(name, N, dt, mixed_tol=3e-8)
    qp, _ = O.sample(31, oracle_system(name), oracle_params(name, N, dt), T, 2500)

    def traced(q):
        tr = np.zeros(4 * 2 * len(q), dtype=np.uint32)
        assert L.hh_cuda_debug_item_trace(tr.ctypes.data, tr.size) == 0
        crln, _ = hh.correlation_from_initial_conditions(ms, p, q, precision)
        return tr.reshape(-1, 4), crln

    tr_all, c_all = traced(qp)
    parts = [traced(qp[c:c + 500]) for c in range(0, 2500, 500)]
    steps = np.concatenate([t[:, 0] for t, _ in parts])
    assert steps.min() > 0
    np.testing.assert_array_equal(tr_all[:, 0], steps)
    np.testing.assert_allclose(sum(c for _, c in parts), c_all, rtol=0, atol=1e-11 * abs(c_all[0]))


def _lib_handle():
    from hawaiihybrid_b200 import _lib
    return _lib.load()


@pytest.mark.parametrize("precision", [0, 1])
def test_traj_tuning_picks_follow_the_same_steps(precision):
    """The autotuner's choices (bulk kernel warps per block, hand-off threshold) change
    only how items are scheduled: every half-trajectory takes the same steps and the
    C(t) agree to rounding, for forced picks and for the autotuner's own (9,000
    CO2-Ar trajectories, above the tuning threshold of 16,384 items)."""
    import hawaiihybrid_b200 as hh
    from hawaiihybrid_b200 import _lib
    ms = lib_system("co2ar")
    L = _lib_handle()
    p = lib_params("co2ar", 256, 100.0, mixed_tol=3e-8)
    qp, _ = O.sample(17, oracle_system("co2ar"), oracle_params("co2ar", 256, 100.0), 300.0, 9000)

    def traced():
        tr = np.zeros(4 * 2 * len(qp), dtype=np.uint32)
        assert L.hh_cuda_debug_item_trace(tr.ctypes.data, tr.size) == 0
        crln, _ = hh.correlation_from_initial_conditions(ms, p, qp, precision)
        return tr.reshape(-1, 4)[:, 0].copy(), crln

    runs = {}
    for w, d in ((4, 1), (8, 1), (8, 4), (4, 2)):
        assert _lib.traj_tuning(precision, w, d) == (w, d)
        runs[(w, d)] = traced()
    _lib.traj_tuning(precision, -1, -1)
    assert _lib.traj_tuning(precision) == (0, 0)
    runs["auto"] = traced()
    w, d = _lib.traj_tuning(precision)
    assert w in (4, 8) and d in (1, 2, 4)
    s0, c0 = runs[(4, 1)]
    assert s0.min() > 0
    for key, (s, c) in runs.items():
        np.testing.assert_array_equal(s, s0, err_msg=str(key))
        np.testing.assert_allclose(c, c0, rtol=0, atol=1e-11 * abs(c0[0]), err_msg=str(key))


@pytest.mark.parametrize("name,integrand,T", [("hear", 0, 100.0), ("co2ar", 0, 100.0), ("co2ar", 1, 300.0),
                                              ("n2ar", 0, 300.0)])
def test_vegas_matches_oracle(name, integrand, T):
    """VEGAS (c_mpi_perform_integration) on the device against the oracle's restatement on
    the same Philox samples: six iterations of 40,000 points, the grid refined between
    them; the grids differ only by the rounding of the per-bin sums."""
    import hawaiihybrid_b200 as hh
    ms = lib_system(name)
    p = lib_params(name, 64, 100.0)
    m, q = hh.c_mpi_perform_integration(ms, integrand, p, T, 6, 40_000, seed=11)
    mr, qr = O.vegas(oracle_system(name), oracle_params(name, 64, 100.0), integrand, T, 6, 40_000, 11)
    assert m > 0 and q > 0
    np.testing.assert_allclose(m, mr, rtol=1e-8)
    np.testing.assert_allclose(q, qr, rtol=1e-6)


@pytest.mark.parametrize("name,published,rel", [("co2ar", 6.25651e-4, 0.01), ("hear", 2.08597e-6, 0.005)])
def test_vegas_m0_published_values(name, published, rel):
    """The reference driver's VEGAS M0 (12 iterations, 1e6 points, scaled by ZeroCoeff /
    pf_analytic) at 100 K reproduces the published values within their accuracy."""
    import hawaiihybrid_b200 as hh
    ms = lib_system(name)
    m0, err = hh.calculate_m0_vegas(ms, lib_params(name, 64, 100.0), 100.0, 12, 1_000_000, seed=3)
    assert abs(m0 - published) <= rel * published + 3 * err


def test_fp64_correlation_at_workload_size():
    """The FP64 path against the oracle at the CO2-Ar workload's sizes: 256 of its
    trajectories (seed 7, 300 K) with all 32,768 samples at dt = 100 a.u.  Both integrate
    the same physics in different coordinates (Cartesian here, the reference's spherical
    ones in the oracle), so late samples of orbiting pairs part chaotically.  Within the
    FP64 horizon (where the device's FP64 runs at rtol 1e-12 and 1e-13 agree to 1e-8 of
    C(0)) they agree to 1e-7 of C(0), and C(0) itself to 1e-12."""
    import hawaiihybrid_b200 as hh
    N, dt = 32768, 100.0
    ms = lib_system("co2ar")
    qp, _ = O.sample(7, oracle_system("co2ar"), oracle_params("co2ar", N, dt), 300.0, 256)
    c12, _ = hh.correlation_from_initial_conditions(ms, lib_params("co2ar", N, dt), qp)
    c13, _ = hh.correlation_from_initial_conditions(ms, lib_params("co2ar", N, dt, tol=1e-13), qp)
    ref = O.correlation_sum(oracle_system("co2ar"), oracle_params("co2ar", N, dt), qp)
    c0 = abs(ref[0])
    floor = np.maximum.accumulate(np.abs(c13 - c12) / c0)
    kh = int(np.argmax(floor > 1e-8)) if np.any(floor > 1e-8) else N
    assert kh > 1000
    assert abs(c12[0] - ref[0]) <= 1e-12 * c0
    assert np.max(np.abs(c12[:kh] - ref[:kh])) <= 1e-7 * c0
