"""CORRELATION_ARRAY (src/hawaii.c:2361-2793) on the GPU against the CPU oracle.

Trajectories are sampled at a base temperature; each adds its C_i(t) to every
satellite temperature's C(t) with the weight exp(-E HkT/T0/Ts (T0-Ts)) / WTT
times that satellite's partial partition function ratio (hawaii.c:2640-2676)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import lib_params, lib_system, oracle_params, oracle_system

pytestmark = pytest.mark.gpu


def _oracle_array(name, seed, T0, Ts, ratios, n, N, dt, ps):
    sysd = oracle_system(name)
    op = oracle_params(name, N, dt, ps=ps)
    qp, _ = O.sample(seed, sysd, op, T0, n)
    w = np.array([O.array_weights(ps, op.pesmin, T0, Ts, O.hamiltonian(sysd, q)) for q in qp])
    data = O.correlation_sum_array(sysd, op, qp, w * np.asarray(ratios)[None, :])
    return data, w.sum(axis=0)


@pytest.mark.parametrize("name,ps,T0,Ts", [
    ("hear", 1, 300.0, [150.0, 250.0, 300.0, 400.0]),
    ("hear", 2, 200.0, [100.0, 200.0, 300.0]),
    ("co2ar", 1, 300.0, [200.0, 300.0]),
])
def test_array_matches_oracle(name, ps, T0, Ts):
    import hawaiihybrid_b200 as hh
    N, dt, n, seed = 1024, 200.0 if name == "hear" else 100.0, 96, 17
    ratios = [1.0 + 0.1 * i for i in range(len(Ts))]
    ms = lib_system(name, seed)
    p = lib_params(name, N, dt, ps=ps)
    p.satellite_temperatures = Ts
    p.partial_partition_function_ratios = ratios
    data, nstar, ntraj, st = hh.correlation_array_iteration(ms, p, T0, n, hh.PRECISION_FP64, seed=seed)
    ref, nstar_ref = _oracle_array(name, seed, T0, Ts, ratios, n, N, dt, ps)
    assert ntraj == n and st.n_failed == 0
    np.testing.assert_allclose(nstar, nstar_ref, rtol=1e-12, atol=0)
    for s in range(len(Ts)):
        scale = max(abs(ref[s][0]), abs(data[s][0]), 1e-300)
        if ps == 1 and Ts[s] > T0:
            assert np.all(data[s] == 0.0) and nstar[s] == 0.0
            continue
        assert np.max(np.abs(data[s] - ref[s])) <= 1e-7 * scale


def test_single_satellite_at_base_equals_plain_correlation():
    import hawaiihybrid_b200 as hh
    ms = lib_system("co2ar", 23)
    p = lib_params("co2ar", 2048, 100.0, ppf=2.5)
    p.satellite_temperatures = [300.0]
    p.partial_partition_function_ratios = [2.5]
    data, nstar, ntraj, _ = hh.correlation_array_iteration(ms, p, 300.0, 512, hh.PRECISION_FP64, seed=23)
    plain, nt, _ = hh.correlation_iteration(ms, p, 300.0, 512, hh.PRECISION_FP64, seed=23)
    assert nstar[0] == 512.0 and ntraj == nt
    np.testing.assert_allclose(data[0], plain, rtol=1e-12, atol=1e-12 * abs(plain[0]))


def test_array_rejects_unsupported_requests():
    import hawaiihybrid_b200 as hh
    ms = lib_system("hear", 3)
    p = lib_params("hear", 64, 200.0, ps=3)
    p.satellite_temperatures = [300.0]
    p.partial_partition_function_ratios = [1.0]
    with pytest.raises(hh.HHError):
        hh.correlation_array_iteration(ms, p, 300.0, 16, hh.PRECISION_FP64, seed=3)
