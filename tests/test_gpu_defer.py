"""Deferred sample evaluation of the mixed path's plain C(t): the trajectory kernel writes
one dense-output context per step and tests only R > Rcut; the sample kernels evaluate the
dipoles, accumulate C(t) and apply the per-sample tests (src/hawaii.c:2183-2243).  Checked
against the in-kernel placement on the same trajectories: the same steps, samples and
statuses, C(t) equal up to the order of the FP64 sums (N2-Ar) or to FP32 rounding (CO2-Ar:
the sample kernel has its own FP32 interpolation and dipole-surface code, with the sample
position in FP32, so a sample's dipole may differ by a few ulps), the same failure handling,
and the same result when the iterations of a call are split over several launches or the
context buffer overflows.  Also: the bulk kernel's per-round block barrier and the sample
launch beside the solo launch change no result."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import lib_params, lib_system, oracle_params, oracle_system, rel_to_c0

pytestmark = pytest.mark.gpu

STAT_KEYS = ("n_steps", "n_rejected_steps", "n_rhs", "n_samples", "n_dense", "n_failed")


@pytest.fixture
def lib():
    from hawaiihybrid_b200 import _lib
    return _lib.load()


def _in_kernel_then_deferred(fn):
    """fn() with the dipoles in the trajectory kernel, then deferred (CO2-Ar and N2-Ar)."""
    from hawaiihybrid_b200 import _lib
    prev = _lib.defer_samples(-1)
    try:
        _lib.defer_samples(0)
        a = fn()
        _lib.defer_samples(2)
        b = fn()
    finally:
        _lib.defer_samples(prev)
    return a, b


def _same_stats(sa, sb):
    for k in STAT_KEYS:
        assert getattr(sa, k) == getattr(sb, k), k
    assert list(sa.status) == list(sb.status)


# C(t) agreement of the two placements, in units of C(0)
PLACEMENT_TOL = {"co2ar": 1e-6, "n2ar": 1e-12}


@pytest.mark.parametrize("name", ["co2ar", "n2ar"])
def test_deferred_samples_match_in_kernel(name):
    import hawaiihybrid_b200 as hh
    ms = lib_system(name, 5)
    N, dt = 4096, 100.0
    qp, _ = O.sample(5, oracle_system(name), oracle_params(name, N, dt), 300.0, 2048)
    p = lib_params(name, N, dt, mixed_tol=3e-8)
    (ca, sa), (cb, sb) = _in_kernel_then_deferred(
        lambda: hh.correlation_from_initial_conditions(ms, p, qp, hh.PRECISION_MIXED))
    assert rel_to_c0(cb, ca) < PLACEMENT_TOL[name]
    _same_stats(sa, sb)


@pytest.mark.parametrize("status", [3, 5])
def test_deferred_failure_matches_in_kernel(lib, status):
    """A hard failure injected at one sample drops the whole trajectory in both placements."""
    import hawaiihybrid_b200 as hh
    name, N, dt = "co2ar", 2048, 100.0
    ms = lib_system(name, 7)
    qp, _ = O.sample(7, oracle_system(name), oracle_params(name, N, dt), 300.0, 256)
    p = lib_params(name, N, dt, mixed_tol=3e-8)
    assert lib.hh_cuda_debug_inject(5, 0, 3, status) == 0
    try:
        (ca, sa), (cb, sb) = _in_kernel_then_deferred(
            lambda: hh.correlation_from_initial_conditions(ms, p, qp, hh.PRECISION_MIXED))
    finally:
        lib.hh_cuda_debug_inject(-1, 0, 0, 0)
    assert sa.n_failed == 1 and sb.n_failed == 1
    assert rel_to_c0(cb, ca) < PLACEMENT_TOL[name]


@pytest.mark.parametrize("name", ["co2ar", "n2ar"])
def test_sample_launch_beside_solo_launch_changes_nothing(lib, name):
    """The contexts of the bulk trajectory launch evaluated while the solo launch runs (the
    default) or after it: the same steps, samples and statuses, C(t) equal up to the
    order of the FP64 sums, a trajectory failed by injection dropped in both."""
    import hawaiihybrid_b200 as hh
    from hawaiihybrid_b200 import _lib
    ms = lib_system(name, 5)
    N, dt = 4096, 100.0
    qp, _ = O.sample(5, oracle_system(name), oracle_params(name, N, dt), 300.0, 2048)
    p = lib_params(name, N, dt, mixed_tol=3e-8)
    prev_d = _lib.defer_samples(2)
    prev_o = _lib.defer_overlap(-1)
    assert lib.hh_cuda_debug_inject(900, 0, 3, 5) == 0
    try:
        out = []
        for on in (0, 1):
            _lib.defer_overlap(on)
            out.append(hh.correlation_from_initial_conditions(ms, p, qp, hh.PRECISION_MIXED))
    finally:
        lib.hh_cuda_debug_inject(-1, 0, 0, 0)
        _lib.defer_overlap(prev_o)
        _lib.defer_samples(prev_d)
    (ca, sa), (cb, sb) = out
    assert sa.n_failed == 1
    assert rel_to_c0(cb, ca) < 1e-12
    _same_stats(sa, sb)
    assert list(sa.status) == list(sb.status)


def test_deferred_launch_split_and_overflow(monkeypatch):
    """Iterations of one call split over several launches (a small context budget), and a
    first context estimate far too small (the call repeats with a larger buffer), give
    the C(t) and statistics of one deferred launch."""
    import hawaiihybrid_b200 as hh
    from hawaiihybrid_b200 import _lib
    ms = lib_system("co2ar", 13)
    p = lib_params("co2ar", 2048, 100.0, mixed_tol=3e-8)
    prev = _lib.defer_samples(1)
    try:
        c1, nt1, s1 = hh.correlation_iterations(ms, p, 300.0, 1000, 4, hh.PRECISION_MIXED, seed=13)
        monkeypatch.setenv("HH_DEFER_BUDGET_MB", "2")
        c2, nt2, s2 = hh.correlation_iterations(ms, p, 300.0, 1000, 4, hh.PRECISION_MIXED, seed=13)
        monkeypatch.delenv("HH_DEFER_BUDGET_MB")
        monkeypatch.setenv("HH_DEFER_EST", "0.5")
        c3, nt3, s3 = hh.correlation_iterations(ms, p, 300.0, 1000, 4, hh.PRECISION_MIXED, seed=13)
        monkeypatch.delenv("HH_DEFER_EST")
    finally:
        _lib.defer_samples(prev)
    for c in (c2, c3):
        for i in range(4):
            assert rel_to_c0(c[i], c1[i]) < 1e-12
    for s in (s2, s3):
        _same_stats(s1, s)
    assert list(nt1) == list(nt2) == list(nt3)


@pytest.mark.parametrize("name,precision", [("hear", 0), ("hear", 1), ("co2ar", 0), ("co2ar", 1),
                                            ("n2ar", 0), ("n2ar", 1), ("ch4co2", 1)])
def test_block_barrier_changes_nothing(monkeypatch, name, precision):
    """The bulk kernel with and without its per-round block barrier integrates the same
    steps and gives the same C(t) (up to the order of the FP64 sums)."""
    import hawaiihybrid_b200 as hh
    ms = lib_system(name, 9)
    N, dt = (21, 200.0) if name == "ch4co2" else (2048, 100.0)
    qp, _ = O.sample(9, oracle_system(name), oracle_params(name, N, dt), 300.0, 1024)
    p = lib_params(name, N, dt, mixed_tol=3e-8)
    out = []
    for bs in ("0", "1"):
        monkeypatch.setenv("HH_TRAJ_BLOCK_SYNC", bs)
        out.append(hh.correlation_from_initial_conditions(ms, p, qp, precision))
    (ca, sa), (cb, sb) = out
    assert rel_to_c0(cb, ca) < 1e-12
    _same_stats(sa, sb)
