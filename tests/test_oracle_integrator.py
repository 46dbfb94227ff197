"""The oracle's FP64 DOP853 + dense output stands in for CVODE (SUNDIALS is not
available): pinned against converged solutions, an independent integrator
(SciPy's DOP853 at rtol 1e-13) and energy conservation."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import oracle_params, oracle_system


@pytest.mark.parametrize("name,dt,seed", [("hear", 200.0, 42), ("co2ar", 100.0, 7)])
def test_states_match_converged_solution(name, dt, seed):
    """states at t = 1000 a.u. within 1e-9 relative of a 100x tighter integration."""
    sysd = oracle_system(name)
    qp, _ = O.sample(seed, sysd, oracle_params(name, 64, dt), 300.0, 8)
    for q in qp:
        a, _ = O.propagate(sysd, oracle_params(name, 64, dt, tol=1e-12), q, 1000.0)
        b, _ = O.propagate(sysd, oracle_params(name, 64, dt, tol=1e-14), q, 1000.0)
        ca, cb = O.qp_to_cart(sysd, a), O.qp_to_cart(sysd, b)
        assert np.max(np.abs(ca - cb) / np.maximum(np.abs(cb), 1.0)) < 1e-9


@pytest.mark.parametrize("name,dt", [("hear", 200.0), ("co2ar", 100.0)])
def test_states_match_scipy_dop853(name, dt):
    from scipy.integrate import solve_ivp
    L = O.lib()
    sysd = oracle_system(name)
    qp, _ = O.sample(3, sysd, oracle_params(name, 64, dt), 300.0, 4)

    def f(t, y):
        out = np.zeros_like(y)
        L.hho_rhs(C.byref(sysd), np.ascontiguousarray(y), out)
        return out
    for q in qp:
        a, _ = O.propagate(sysd, oracle_params(name, 64, dt), q, 1000.0)
        s = solve_ivp(f, (0.0, 1000.0), q, method="DOP853", rtol=1e-13, atol=1e-13)
        ca, cb = O.qp_to_cart(sysd, a), O.qp_to_cart(sysd, s.y[:, -1])
        assert np.max(np.abs(ca - cb) / np.maximum(np.abs(cb), 1.0)) < 1e-9


@pytest.mark.parametrize("name,dt", [("hear", 200.0), ("co2ar", 100.0)])
def test_energy_conservation(name, dt):
    """|E - E0| <= 1000 rtol along trajectories (src/trajectory.c:167-180)."""
    L = O.lib()
    sysd = oracle_system(name)
    qp, _ = O.sample(11, sysd, oracle_params(name, 64, dt), 300.0, 6)
    for q in qp:
        E0 = L.hho_hamiltonian(C.byref(sysd), q)
        y, _ = O.propagate(sysd, oracle_params(name, 64, dt), q, 50000.0)
        E1 = L.hho_hamiltonian(C.byref(sysd), y)
        assert abs(E1 - E0) <= 1000 * 1e-12


def test_correlation_eval_structure():
    """crln[0] = |mu0|^2 ALU^3, exits at R > Rcut leave zeros, branches are symmetric."""
    sysd = oracle_system("hear")
    p = oracle_params("hear", 4096, 200.0)
    qp, _ = O.sample(42, sysd, p, 300.0, 4)
    for q in qp:
        crln, st = O.correlation_eval(sysd, p, q)
        fw, bw = O.correlation_parts(sysd, p, q)
        assert st.failed == 0 and st.status_fwd == 0 and st.status_bwd == 0
        d = np.zeros(3)
        O.lib().hho_dipole(C.byref(sysd), np.ascontiguousarray(q[::2]), d)
        assert crln[0] == pytest.approx(np.dot(d, d) * 5.29177210903e-11 ** 3, rel=1e-14)
        last = max(np.nonzero(fw)[0].max(), np.nonzero(bw)[0].max())
        assert np.all(crln[last + 1:] == 0.0)
        np.testing.assert_allclose(crln, 0.5 * (fw + bw) * 5.29177210903e-11 ** 3, rtol=1e-15, atol=0)


def test_sampler_draw_counts_and_filter():
    """D = 10 (atom-atom) / 16 (linear-atom) words per candidate; accepted free states have H >= 0."""
    L = O.lib()
    for name, D in (("hear", 10), ("co2ar", 16)):
        sysd = oracle_system(name)
        p = oracle_params(name, 64, 100.0)
        s = O.lib()
        mt = (C.c_uint32 * 625)()
        st = C.create_string_buffer(C.sizeof(C.c_uint32) * 626)
        qp, cand = O.sample(5, sysd, p, 300.0, 200)
        for q in qp:
            assert L.hho_hamiltonian(C.byref(sysd), q) >= 0.0
        # the accepted set is a prefix-consistent function of the stream
        qp2, cand2 = O.sample(5, sysd, p, 300.0, 100)
        np.testing.assert_array_equal(qp2, qp[:100])
        assert cand2 <= cand
