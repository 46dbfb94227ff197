"""N2-Ar PIP-NN on the GPU against the CPU oracle, through the C ABI (libhh_cuda.so).

Workload shapes follow the reference's N2-Ar example (examples/correlation_n2_ar.cpp:
sampler R in [4.51, 40], pesmin -97.3 cm^-1, Rcut 40), at sizes the oracle
finishes in seconds."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import lib_params, lib_system, oracle_params, oracle_system, rel_to_c0

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed,T,n", [(7, 200.0, 2000), (20106943, 300.0, 1000)])
def test_sampler_matches_oracle(seed, T, n):
    import hawaiihybrid_b200 as hh
    ms = lib_system("n2ar", seed)
    p = lib_params("n2ar", 64, 100.0)
    qp, cand = hh.sample_initial_conditions(ms, p, T, n, seed=seed)
    qp_ref, cand_ref = O.sample(seed, oracle_system("n2ar"), oracle_params("n2ar", 64, 100.0), T, n)
    assert cand == cand_ref
    np.testing.assert_allclose(qp, qp_ref, rtol=1e-13, atol=1e-300)


def test_single_trajectory_early_times():
    """Per-trajectory C_i(t_k) over the first 2000 a.u., 1e-9 of C_i(0): checks the device
    PES gradient (forces and torques) and the dipole against the oracle's lab-frame path."""
    import hawaiihybrid_b200 as hh
    ms = lib_system("n2ar")
    dt = 100.0
    qp, _ = O.sample(9, oracle_system("n2ar"), oracle_params("n2ar", 64, dt), 200.0, 16)
    kmax = int(2000.0 / dt) + 1
    for i in range(qp.shape[0]):
        crln, _ = hh.correlation_from_initial_conditions(ms, lib_params("n2ar", 64, dt), qp[i:i + 1])
        ref, st = O.correlation_eval(oracle_system("n2ar"), oracle_params("n2ar", 64, dt), qp[i])
        assert np.max(np.abs(crln[:kmax] - ref[:kmax])) <= 1e-9 * abs(ref[0])


def test_fp64_correlation_matches_oracle():
    import hawaiihybrid_b200 as hh
    N, dt, n = 2048, 100.0, 96
    ms = lib_system("n2ar")
    qp, _ = O.sample(42, oracle_system("n2ar"), oracle_params("n2ar", N, dt), 200.0, n)
    crln, st = hh.correlation_from_initial_conditions(ms, lib_params("n2ar", N, dt), qp)
    ref = O.correlation_sum(oracle_system("n2ar"), oracle_params("n2ar", N, dt), qp)
    assert st.n_failed == 0
    assert rel_to_c0(crln, ref) < 1e-7


def test_mixed_matches_fp64():
    """Mixed (FP32 surfaces) against FP64 on the same initial conditions: M0 from C(0) to
    1e-6 and C(t) to 1e-4 of C(0) over t <= 1e5 a.u."""
    import hawaiihybrid_b200 as hh
    ms = lib_system("n2ar")
    p = lib_params("n2ar", 4096, 100.0)
    c64, _, s64 = hh.correlation_iteration(ms, p, 200.0, 1024, hh.PRECISION_FP64, seed=5)
    c32, _, s32 = hh.correlation_iteration(ms, p, 200.0, 1024, hh.PRECISION_MIXED, seed=5)
    assert rel_to_c0(c32[:1001], c64[:1001]) <= 1e-4
    assert abs(c32[0] - c64[0]) / abs(c64[0]) <= 1e-6


def test_m0_matches_oracle():
    import hawaiihybrid_b200 as hh
    ms = lib_system("n2ar")
    p = lib_params("n2ar", 64, 100.0)
    T = np.array([150.0, 200.0, 300.0])
    n = 1 << 16
    m64, e64 = hh.calculate_m0(ms, p, T, n, seed=99, precision=hh.PRECISION_FP64)
    m32, _ = hh.calculate_m0(ms, p, T, n, seed=99, precision=hh.PRECISION_MIXED)
    ws, wq = O.m0(oracle_system("n2ar"), oracle_params("n2ar", 64, 100.0), T, n, 99)
    mref = O.m0_scale(oracle_params("n2ar", 64, 100.0)) * ws / n
    np.testing.assert_allclose(m64, mref, rtol=1e-10)
    np.testing.assert_allclose(m32, m64, rtol=1e-4)
    assert np.all(e64 > 0) and np.all(e64 < 0.1 * m64)


def test_mixed_dipole_table_matches_network():
    """The mixed path's FP32 dipole table against the FP64 network (itself checked
    against the oracle here): within 2e-6 of the largest |d| over T at the same R,
    inside the table's range [4.5, 60) bohr and across its cell edges; outside it the
    mixed path evaluates the network."""
    import hawaiihybrid_b200 as hh
    from hawaiihybrid_b200 import _lib
    lib_system("n2ar")
    L = _lib.load()
    rng = np.random.default_rng(11)
    n = 1500
    R = np.concatenate([rng.uniform(4.5, 60.0, n), np.array([4.5, 9.5, 12.5, 20.0, 59.999]),
                        rng.uniform(3.8, 4.5, 20), rng.uniform(60.0, 80.0, 20)])
    T = np.concatenate([rng.uniform(0.0, np.pi, n), np.array([0.0, np.pi / 12, np.pi / 2, np.pi, 1e-4]),
                        rng.uniform(0.0, np.pi, 40)])
    m = len(R)
    Tg = np.linspace(0.0, np.pi, 25)
    Rs = np.repeat(R, len(Tg))
    Ts = np.tile(Tg, m)

    def dip(prec, r, t):
        out = np.zeros(2 * len(r))
        _lib.check(L.hh_cuda_debug_n2ar_dipole(prec, np.ascontiguousarray(r), np.ascontiguousarray(t), len(r), out))
        return out.reshape(-1, 2)

    d64 = dip(hh.PRECISION_FP64, R, T)
    d32 = dip(hh.PRECISION_MIXED, R, T)
    scale = np.abs(dip(hh.PRECISION_FP64, Rs, Ts)).reshape(m, -1).max(axis=1)
    for i in range(0, m, 97):
        ref = O.n2ar_dip_mol(R[i], T[i])
        # the network's output is a difference of O(0.1) charges: about 1e-15 bohr e absolute
        np.testing.assert_allclose(d64[i], [ref[0], ref[2]], rtol=0, atol=1e-14 + 1e-9 * scale[i])
    err = np.abs(d32 - d64).max(axis=1) / scale
    assert err.max() < 2e-6, (err.max(), R[np.argmax(err)], T[np.argmax(err)])
    outside = (R < 4.5) | (R >= 60.0)
    np.testing.assert_allclose(d32[outside], d64[outside], rtol=0, atol=1e-12)


@pytest.mark.parametrize("precision", [0, 1])
def test_solo_kernel_follows_the_bulk_path(precision):
    """The last open items of a launch move to the solo kernel (one warp per item,
    the PES network shared by the lanes); a launch with no more items than warp
    slots runs there from the start.  The cooperative right-hand side is
    bit-identical to the per-lane one, so every half-trajectory takes the same steps
    either way: a 1500-trajectory launch (bulk, then hand-off) against the same
    trajectories in three launches of 500 (solo only), per item, and the sum of
    their C(t) against its C(t)."""
    import hawaiihybrid_b200 as hh
    from hawaiihybrid_b200 import _lib
    ms = lib_system("n2ar")
    L = _lib.load()
    p = lib_params("n2ar", 2048, 100.0, mixed_tol=3e-8)
    qp, _ = O.sample(31, oracle_system("n2ar"), oracle_params("n2ar", 2048, 100.0), 200.0, 1500)

    def traced(q):
        tr = np.zeros(4 * 2 * len(q), dtype=np.uint32)
        _lib.check(L.hh_cuda_debug_item_trace(tr.ctypes.data, tr.size))
        crln, st = hh.correlation_from_initial_conditions(ms, p, q, precision)
        return tr.reshape(-1, 4), crln

    tr_all, c_all = traced(qp)
    parts = [traced(qp[c:c + 500]) for c in range(0, 1500, 500)]
    steps = np.concatenate([t[:, 0] for t, _ in parts])
    assert steps.min() > 0
    np.testing.assert_array_equal(tr_all[:, 0], steps)   # accepted steps per item
    c_sum = sum(c for _, c in parts)
    np.testing.assert_allclose(c_sum, c_all, rtol=0, atol=1e-11 * abs(c_all[0]))
