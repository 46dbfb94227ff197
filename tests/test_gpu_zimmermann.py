"""Zimmermann's estimate (correlation_eval_zimmerman_trick, src/hawaii.c:1888-2114) on the GPU
against the CPU oracle: for BOUND pairs each trajectory's C_i(s) is
sum_{c < N} d[c].d[c+s] ALU^3 / N over the dipole series d of both branches
(d[N-1] = mu0, d[N-1+k] = mu(t_k), d[N-1-k] = mu(-t_k)), through the C ABI."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import lib_params, lib_system, oracle_params, oracle_system, rel_to_c0

pytestmark = pytest.mark.gpu

CASES = [("hear", 50.0, 200.0, 256), ("co2ar", 100.0, 100.0, 256), ("n2ar", 80.0, 100.0, 128),
         ("ch4co2", 100.0, 200.0, 100)]


def _params(name, N, dt):
    p = lib_params(name, N, dt, ps=2)
    p.use_zimmermann_trick = True
    return p


@pytest.mark.parametrize("name,T,dt,N", CASES)
def test_fp64_matches_oracle(name, T, dt, N):
    import hawaiihybrid_b200 as hh
    ms = lib_system(name)
    op = oracle_params(name, N, dt, ps=O.PS_BOUND)
    qp, _ = O.sample(3, oracle_system(name), op, T, 48)
    crln, st = hh.correlation_from_initial_conditions(ms, _params(name, N, dt), qp)
    op.zimmermann = 1
    ref = O.correlation_sum(oracle_system(name), op, qp)
    assert st.n_failed == 0
    assert rel_to_c0(crln, ref) < 1e-8


@pytest.mark.parametrize("name,T,dt,N", [CASES[1], CASES[3]])
def test_mixed_matches_fp64(name, T, dt, N):
    import hawaiihybrid_b200 as hh
    ms = lib_system(name)
    p = _params(name, N, dt)
    c64, _, _ = hh.correlation_iteration(ms, p, T, 512, hh.PRECISION_FP64, seed=9)
    c32, _, _ = hh.correlation_iteration(ms, p, T, 512, hh.PRECISION_MIXED, seed=9)
    assert rel_to_c0(c32, c64) <= 1e-4


def test_single_trajectory_lag_zero():
    """C_i(0) = sum_{c < N} |d[c]|^2 ALU^3 / N: the backward half and mu0 only."""
    import hawaiihybrid_b200 as hh
    name, T, dt, N = "co2ar", 100.0, 100.0, 64
    ms = lib_system(name)
    op = oracle_params(name, N, dt, ps=O.PS_BOUND)
    qp, _ = O.sample(8, oracle_system(name), op, T, 1)
    crln, _ = hh.correlation_from_initial_conditions(ms, _params(name, N, dt), qp)
    ref, _ = O.correlation_eval_zimmermann(oracle_system(name), op, qp[0])
    np.testing.assert_allclose(crln, ref, rtol=1e-9, atol=1e-9 * abs(ref[0]))


def test_requires_bound_pairs():
    import hawaiihybrid_b200 as hh
    ms = lib_system("hear")
    p = lib_params("hear", 64, 200.0, ps=1)
    p.use_zimmermann_trick = True
    with pytest.raises(hh.HHError):
        hh.correlation_iteration(ms, p, 300.0, 16, hh.PRECISION_FP64, seed=1)


def test_fft_long_series_matches_oracle():
    """N = 1000 (transform length 2048, not a multiple of N): the FFT cross-correlation
    against the oracle's direct lagged sum."""
    import hawaiihybrid_b200 as hh
    name, T, dt, N = "hear", 50.0, 200.0, 1000
    ms = lib_system(name)
    op = oracle_params(name, N, dt, ps=O.PS_BOUND)
    qp, _ = O.sample(5, oracle_system(name), op, T, 24)
    crln, st = hh.correlation_from_initial_conditions(ms, _params(name, N, dt), qp)
    op.zimmermann = 1
    ref = O.correlation_sum(oracle_system(name), op, qp)
    assert st.n_failed == 0
    assert rel_to_c0(crln, ref) < 1e-8


def test_iterations_fill_their_slices():
    """Three iterations in one launch: each iteration's lagged sums land in its own C(t)
    slice, and the slices add up to one pass over the same 192 trajectories."""
    import hawaiihybrid_b200 as hh
    ms = lib_system("co2ar")
    p = _params("co2ar", 128, 100.0)
    cs, nt, _ = hh.correlation_iterations(ms, p, 100.0, 64, 3, hh.PRECISION_FP64, seed=4)
    c1, _, _ = hh.correlation_iteration(ms, p, 100.0, 192, hh.PRECISION_FP64, seed=4)
    assert all(abs(cs[i][0]) > 0 for i in range(3))
    np.testing.assert_allclose(cs.sum(axis=0), c1, rtol=0, atol=1e-12 * abs(c1[0]))
