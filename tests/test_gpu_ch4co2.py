"""CH4-CO2 (ROTOR + LINEAR) on the GPU against the CPU oracle, through the C ABI.

Workload shapes follow the reference's CH4-CO2 configuration
(example_configs/CF-F-CH4-CO2.conf: sampler R in [4.751, 40], pesmin
-1.562522273622102e-03, Rcut 40, sampling_time 200, MaxTrajectoryLength 21).  The
trajectories run on the stand-in surface of hh_ch4co2_standin.h (the reference has
no source for its CH4-CO2 PES); the dipole is the reference's own."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import lib_params, lib_system, oracle_params, oracle_system, rel_to_c0

pytestmark = pytest.mark.gpu
N, DT = 21, 200.0


@pytest.mark.parametrize("seed,T,n", [(7, 100.0, 1500), (2066497031, 300.0, 800)])
def test_sampler_matches_oracle(seed, T, n):
    """25 words per candidate: q_generator (3 + 3 + 2), p_generator (3 + 3 + 2 normals), reject."""
    import hawaiihybrid_b200 as hh
    ms = lib_system("ch4co2", seed)
    qp, cand = hh.sample_initial_conditions(ms, lib_params("ch4co2", N, DT), T, n, seed=seed)
    qp_ref, cand_ref = O.sample(seed, oracle_system("ch4co2"), oracle_params("ch4co2", N, DT), T, n)
    assert cand == cand_ref
    # the rotor momenta are three-term sums of sin/cos products, so a last-ulp difference
    # between the device's and the host's sin/cos can reach ~1e-13 of the sum
    np.testing.assert_allclose(qp, qp_ref, rtol=1e-12, atol=1e-300)


@pytest.mark.parametrize("precision,tol", [(0, 1e-12), (1, 2e-5)])
def test_t0_dipoles_match_oracle(precision, tol):
    """N = 1 keeps only C(0) = sum_i |mu_i(0)|^2 ALU^3: the batched dipole kernel over
    400 sampled configurations (every radial piece the sampler reaches)."""
    import hawaiihybrid_b200 as hh
    ms = lib_system("ch4co2")
    qp, _ = O.sample(3, oracle_system("ch4co2"), oracle_params("ch4co2", 1, DT), 400.0, 400)
    ref = O.correlation_sum(oracle_system("ch4co2"), oracle_params("ch4co2", 1, DT), qp)
    for i in range(0, 400, 40):
        c, _ = hh.correlation_from_initial_conditions(ms, lib_params("ch4co2", 1, DT), qp[i:i + 40], precision)
        r = O.correlation_sum(oracle_system("ch4co2"), oracle_params("ch4co2", 1, DT), qp[i:i + 40])
        assert abs(c[0] - r[0]) <= tol * r[0]
    c, _ = hh.correlation_from_initial_conditions(ms, lib_params("ch4co2", 1, DT), qp, precision)
    assert abs(c[0] - ref[0]) <= tol * ref[0]


def test_single_trajectory_early_times():
    """Per-trajectory C_i(t_k) for t <= 2000 a.u. to 1e-9 of C_i(0): the quaternion
    rotor dynamics against the reference's Euler-angle equations."""
    import hawaiihybrid_b200 as hh
    ms = lib_system("ch4co2")
    qp, _ = O.sample(9, oracle_system("ch4co2"), oracle_params("ch4co2", N, DT), 200.0, 12)
    kmax = int(2000.0 / DT) + 1
    for i in range(qp.shape[0]):
        crln, _ = hh.correlation_from_initial_conditions(ms, lib_params("ch4co2", N, DT), qp[i:i + 1])
        ref, st = O.correlation_eval(oracle_system("ch4co2"), oracle_params("ch4co2", N, DT), qp[i])
        assert np.max(np.abs(crln[:kmax] - ref[:kmax])) <= 1e-9 * abs(ref[0])


def test_fp64_correlation_matches_oracle():
    import hawaiihybrid_b200 as hh
    ms = lib_system("ch4co2")
    qp, _ = O.sample(42, oracle_system("ch4co2"), oracle_params("ch4co2", N, DT), 300.0, 128)
    crln, st = hh.correlation_from_initial_conditions(ms, lib_params("ch4co2", N, DT), qp)
    ref = O.correlation_sum(oracle_system("ch4co2"), oracle_params("ch4co2", N, DT), qp)
    assert st.n_failed == 0
    assert rel_to_c0(crln, ref) < 1e-8


def test_rcut_exits_match_oracle():
    """Pairs sampled at R in [34, 40] with N = 100 (20,000 a.u.): most branches leave the
    Rcut sphere after a few samples, so the stored sample count of each branch decides
    which records enter C(t)."""
    import hawaiihybrid_b200 as hh
    ms = lib_system("ch4co2")
    op = oracle_params("ch4co2", 100, DT, Rmin=34.0)
    qp, _ = O.sample(5, oracle_system("ch4co2"), op, 400.0, 16)
    crln, st = hh.correlation_from_initial_conditions(ms, lib_params("ch4co2", 100, DT, Rmin=34.0), qp)
    ref = O.correlation_sum(oracle_system("ch4co2"), op, qp)
    ends = []
    for q in qp:
        fw, bw = O.correlation_parts(oracle_system("ch4co2"), op, q)
        ends += [int(np.max(np.nonzero(fw)[0])), int(np.max(np.nonzero(bw)[0]))]
    assert min(ends) < 99    # some branches leave before the last sample
    assert st.status[0] == 32
    assert rel_to_c0(crln, ref) < 1e-7


def test_immediate_exit_beyond_rcut():
    import hawaiihybrid_b200 as hh
    ms = lib_system("ch4co2")
    op = oracle_params("ch4co2", 64, DT, Rmin=30.0, Rcut=20.0)
    qp, _ = O.sample(5, oracle_system("ch4co2"), op, 300.0, 16)
    crln, st = hh.correlation_from_initial_conditions(ms, lib_params("ch4co2", 64, DT, Rmin=30.0, Rcut=20.0), qp)
    ref = O.correlation_sum(oracle_system("ch4co2"), op, qp)
    assert np.all(ref[2:] == 0.0) and np.all(crln[2:] == 0.0)
    assert rel_to_c0(crln[:2], ref[:2]) < 1e-10


def test_mixed_matches_fp64():
    """Mixed (FP32 surfaces, stages and dipole) against FP64 on the same initial
    conditions: C(t) to 1e-4 of C(0), C(0) (hence M0) to 1e-5."""
    import hawaiihybrid_b200 as hh
    ms = lib_system("ch4co2")
    p = lib_params("ch4co2", N, DT)
    c64, _, _ = hh.correlation_iteration(ms, p, 300.0, 4096, hh.PRECISION_FP64, seed=5)
    c32, _, _ = hh.correlation_iteration(ms, p, 300.0, 4096, hh.PRECISION_MIXED, seed=5)
    assert rel_to_c0(c32, c64) <= 1e-4
    assert abs(c32[0] - c64[0]) / abs(c64[0]) <= 1e-5


def test_temperatures_match_consecutive_samples():
    """hh_cuda_correlation_temperatures equals sampling the temperature sets one after
    another from the same stream and integrating each set."""
    import hawaiihybrid_b200 as hh
    ms = lib_system("ch4co2", 11)
    p = lib_params("ch4co2", N, DT)
    Ts = [100.0, 200.0, 300.0, 400.0]
    c, nt, st = hh.correlation_temperatures(ms, p, Ts, 96, hh.PRECISION_FP64, seed=11)
    assert c.shape == (4, N) and np.all(nt == 96)
    for i, T in enumerate(Ts):
        qp, _ = hh.sample_initial_conditions(ms, p, T, 96, seed=11 if i == 0 else 0)
        ref, _ = hh.correlation_from_initial_conditions(ms, p, qp)
        np.testing.assert_allclose(c[i], ref, rtol=1e-12, atol=1e-12 * abs(ref[0]))


@pytest.mark.parametrize("status,hard", [(3, True), (1, False)])
def test_failure_semantics(status, hard):
    """The record path applies the reference's per-sample tests after the batched dipole:
    a hard failure drops the trajectory, an integrator failure keeps earlier samples."""
    import hawaiihybrid_b200 as hh
    from hawaiihybrid_b200 import _lib
    L = _lib.load()
    ms = lib_system("ch4co2")
    qp, _ = O.sample(21, oracle_system("ch4co2"), oracle_params("ch4co2", N, DT), 300.0, 24)
    traj, k_fail = 5, 3
    assert L.hh_cuda_debug_inject(traj, 0, k_fail, status) == 0
    try:
        crln, st = hh.correlation_from_initial_conditions(ms, lib_params("ch4co2", N, DT), qp)
    finally:
        L.hh_cuda_debug_inject(-1, 0, 0, 0)
    keep = [i for i in range(qp.shape[0]) if i != traj]
    ref = O.correlation_sum(oracle_system("ch4co2"), oracle_params("ch4co2", N, DT), qp[keep])
    if not hard:
        fw, bw = O.correlation_parts(oracle_system("ch4co2"), oracle_params("ch4co2", N, DT), qp[traj])
        fw[k_fail:] = 0.0
        ref = ref + 0.5 * (fw + bw) * (5.29177210903e-11) ** 3
    assert st.n_failed == (1 if hard else 0)
    assert rel_to_c0(crln, ref) < 1e-8


def test_m0_is_rejected():
    import hawaiihybrid_b200 as hh
    ms = lib_system("ch4co2")
    with pytest.raises(hh.HHError):
        hh.calculate_m0(ms, lib_params("ch4co2", N, DT), [300.0], 1 << 12)


def test_dipole_tuner_picks_a_candidate():
    """The first record-path call of a context times the dipole kernel's variants (1, 2, 4
    records per lane and the tensor-core kernel (-1) for FP32; 1, 2 for FP64) and keeps the
    fastest; the C(t) of the tuning call and of a later call on the same trajectories
    agree."""
    import ctypes as C
    import hawaiihybrid_b200 as hh
    from hawaiihybrid_b200 import _lib
    ms = lib_system("ch4co2")
    L = _lib.load()
    p = lib_params("ch4co2", 21, 200.0)
    qp, _ = O.sample(3, oracle_system("ch4co2"), oracle_params("ch4co2", 21, 200.0), 300.0, 256)
    c1, _ = hh.correlation_from_initial_conditions(ms, p, qp, hh.PRECISION_MIXED)
    c2, _ = hh.correlation_from_initial_conditions(ms, p, qp, hh.PRECISION_MIXED)
    s64, s32 = C.c_int(-1), C.c_int(-1)
    assert L.hh_cuda_debug_tuning(C.byref(s64), C.byref(s32)) == 0
    assert s32.value in (1, 2, 4, -1)
    np.testing.assert_allclose(c2, c1, rtol=0, atol=1e-12 * abs(c1[0]))


@pytest.mark.parametrize("variant", [1, 2, 4, -1])
def test_mixed_dipole_variants(variant):  # noqa: selected by -k variants
    """Every variant of the FP32 record-path dipole (1, 2 or 4 records per lane on the
    CUDA cores; -1: the tcgen05 tensor-core kernel, TF32 with a three-product split)
    against the oracle: C(0) over 400 sampled configurations (every radial piece the
    sampler reaches) within 2e-5, and a 600-trajectory C(t) within 1e-4 of C(0) of the
    FP64 path on the same initial conditions."""
    import hawaiihybrid_b200 as hh
    from hawaiihybrid_b200 import _lib
    ms = lib_system("ch4co2")
    L = _lib.load()
    assert L.hh_cuda_debug_set_ch4_dipole(1, variant) == 0
    try:
        qp, _ = O.sample(3, oracle_system("ch4co2"), oracle_params("ch4co2", 1, DT), 400.0, 400)
        ref = O.correlation_sum(oracle_system("ch4co2"), oracle_params("ch4co2", 1, DT), qp)
        c, _ = hh.correlation_from_initial_conditions(ms, lib_params("ch4co2", 1, DT), qp, 1)
        assert abs(c[0] - ref[0]) <= 2e-5 * ref[0]
        qp, _ = O.sample(11, oracle_system("ch4co2"), oracle_params("ch4co2", N, DT), 200.0, 600)
        c64, _ = hh.correlation_from_initial_conditions(ms, lib_params("ch4co2", N, DT), qp, 0)
        c32, _ = hh.correlation_from_initial_conditions(ms, lib_params("ch4co2", N, DT, mixed_tol=3e-8), qp, 1)
        assert rel_to_c0(c32, c64) < 1e-4
        s64, s32 = C.c_int(0), C.c_int(0)
        assert L.hh_cuda_debug_tuning(C.byref(s64), C.byref(s32)) == 0
        assert s32.value == variant
    finally:
        L.hh_cuda_debug_set_ch4_dipole(1, 0)
