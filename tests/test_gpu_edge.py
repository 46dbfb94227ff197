"""Edge cases of the trajectory path on the GPU against the oracle: a single
trajectory, the shortest C(t) (MaxTrajectoryLength 1 and 2), trajectories that
leave the Rcut sphere at once, the mixed path of CORRELATION_ARRAY, and argument
checks at the C ABI."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import lib_params, lib_system, oracle_params, oracle_system, rel_to_c0

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["hear", "co2ar", "n2ar"])
@pytest.mark.parametrize("N", [1, 2, 3])
def test_shortest_trajectories(name, N):
    """N = 1 keeps only the t = 0 term; N = 2 and 3 stop after one and two samples."""
    import hawaiihybrid_b200 as hh
    dt = 200.0 if name == "hear" else 100.0
    ms = lib_system(name)
    qp, _ = O.sample(31, oracle_system(name), oracle_params(name, N, dt), 300.0, 8)
    crln, st = hh.correlation_from_initial_conditions(ms, lib_params(name, N, dt), qp)
    ref = O.correlation_sum(oracle_system(name), oracle_params(name, N, dt), qp)
    assert crln.shape == (N,)
    assert rel_to_c0(crln, ref) < 1e-9


@pytest.mark.parametrize("name", ["hear", "co2ar"])
def test_single_trajectory_whole_run(name):
    import hawaiihybrid_b200 as hh
    N, dt = 4096, 200.0 if name == "hear" else 100.0
    ms = lib_system(name)
    qp, _ = O.sample(77, oracle_system(name), oracle_params(name, N, dt), 300.0, 1)
    crln, st = hh.correlation_from_initial_conditions(ms, lib_params(name, N, dt), qp)
    ref, rst = O.correlation_eval(oracle_system(name), oracle_params(name, N, dt), qp[0])
    assert st.n_failed == rst.failed == 0
    assert rel_to_c0(crln, ref) < 1e-7


@pytest.mark.parametrize("name", ["hear", "co2ar"])
def test_immediate_exit_beyond_rcut(name):
    """With Rcut below the sampled separations every branch stores sample 1 and stops
    (the exit test follows the store, src/hawaii.c:2243)."""
    import hawaiihybrid_b200 as hh
    N, dt = 256, 200.0 if name == "hear" else 100.0
    ms = lib_system(name)
    op = oracle_params(name, N, dt, Rmin=30.0, Rcut=20.0)
    qp, _ = O.sample(5, oracle_system(name), op, 300.0, 16)
    crln, st = hh.correlation_from_initial_conditions(ms, lib_params(name, N, dt, Rmin=30.0, Rcut=20.0), qp)
    ref = O.correlation_sum(oracle_system(name), op, qp)
    assert np.all(ref[2:] == 0.0) and np.all(crln[2:] == 0.0)
    assert rel_to_c0(crln[:2], ref[:2]) < 1e-9


def test_array_mixed_matches_fp64():
    import hawaiihybrid_b200 as hh
    ms = lib_system("co2ar", 19)
    p = lib_params("co2ar", 2048, 100.0)
    p.satellite_temperatures = [250.0, 300.0]
    p.partial_partition_function_ratios = [1.0, 1.0]
    d64, n64, _, _ = hh.correlation_array_iteration(ms, p, 300.0, 512, hh.PRECISION_FP64, seed=19)
    d32, n32, _, _ = hh.correlation_array_iteration(ms, p, 300.0, 512, hh.PRECISION_MIXED, seed=19)
    np.testing.assert_array_equal(n32, n64)   # the weights come from the same FP64 energies
    for s in range(2):
        assert rel_to_c0(d32[s][:1001], d64[s][:1001]) <= 1e-4


def test_abi_rejects_bad_arguments():
    from hawaiihybrid_b200 import _lib
    L = _lib.load()
    lib_system("hear")
    cp = lib_params("hear", 64, 200.0).to_c()
    out = np.zeros(64)
    nt = C.c_double()
    st = _lib.Stats()
    # zero trajectories, non-positive temperature, unknown precision
    assert L.hh_cuda_correlation(C.byref(cp), 300.0, 1, 0, 0, out, C.byref(nt), C.byref(st)) == _lib.HH_E_INVALID_ARGUMENT
    assert L.hh_cuda_correlation(C.byref(cp), -1.0, 1, 8, 0, out, C.byref(nt), C.byref(st)) == _lib.HH_E_INVALID_ARGUMENT
    assert L.hh_cuda_correlation(C.byref(cp), 300.0, 1, 8, 7, out, C.byref(nt), C.byref(st)) == _lib.HH_E_INVALID_ARGUMENT
    # an inverted sampler range
    bad = lib_params("hear", 64, 200.0, Rmin=40.0, Rmax=4.0).to_c()
    assert L.hh_cuda_correlation(C.byref(bad), 300.0, 1, 8, 0, out, C.byref(nt), C.byref(st)) == _lib.HH_E_INVALID_ARGUMENT
    # the CF -> SF transform needs a power of two
    cf = np.ones(100)
    assert L.hh_cuda_idct_cf_to_sf(cf, 100, 200.0, np.zeros(100), np.zeros(100)) == _lib.HH_E_NOT_POWER_OF_TWO
