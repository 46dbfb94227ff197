"""CH4-CO2 pieces of the CPU oracle: the dipole chain against the reference's own
code (golden fixture from PES-IDS/ai_ids_ch4_co2.cpp, ai_ids_ch4_co2_lib.cpp and
src/angles_handler.cpp compiled in oracle/_ref), and the stand-in potential."""
import os

import numpy as np

from oracle import oracle as O
from tests.helpers import PESMIN_CH4CO2, oracle_params, oracle_system

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_ch4co2_dipole.npz")


def test_dipole_chain_matches_reference_golden():
    g = np.load(GOLDEN)
    sysd = oracle_system("ch4co2")
    for i in range(g["q"].shape[0]):
        kal = O.ch4co2_lab_to_kal(g["q"][i])
        assert np.max(np.abs(kal - g["kal"][i])) <= 1e-13
        dk = O.ch4co2_dipole_kal(g["kal"][i])
        scale = max(np.max(np.abs(g["dip_kal"][i])), 1e-300)
        assert np.max(np.abs(dk - g["dip_kal"][i])) <= 1e-12 * scale
        dl = O.dipole(sysd, g["q"][i])
        assert np.max(np.abs(dl - g["dip_lab"][i])) <= 1e-12 * scale


def test_standin_gradient_matches_finite_differences():
    sysd = oracle_system("ch4co2")
    rng = np.random.default_rng(11)
    for _ in range(10):
        q = np.array([rng.uniform(0, 6.28), rng.uniform(0.2, 2.9), rng.uniform(6, 12), rng.uniform(0, 6.28),
                      rng.uniform(0.2, 2.9), rng.uniform(0, 6.28), rng.uniform(0, 6.28), rng.uniform(0.2, 2.9)])
        g = O.dpes(sysd, q)
        for k in range(8):
            h = 1e-5
            qp, qm = q.copy(), q.copy()
            qp[k] += h
            qm[k] -= h
            fd = (O.pes(sysd, qp) - O.pes(sysd, qm)) / (2 * h)
            assert abs(fd - g[k]) <= 1e-7 * np.max(np.abs(g))


def test_standin_minimum_is_pesmin():
    """The stand-in is scaled so that its global minimum is the configuration's pesmin."""
    from scipy.optimize import minimize
    sysd = oracle_system("ch4co2")
    rng = np.random.default_rng(3)
    best = 0.0
    for _ in range(24):
        x0 = np.array([rng.uniform(0, 6.28), rng.uniform(0.2, 2.9), rng.uniform(5.8, 7.5), rng.uniform(0, 6.28),
                       rng.uniform(0.2, 2.9), rng.uniform(0, 6.28), rng.uniform(0, 6.28), rng.uniform(0.2, 2.9)])
        r = minimize(lambda q: O.pes(sysd, q), x0, jac=lambda q: O.dpes(sysd, q), method="BFGS",
                     options={"gtol": 1e-12})
        best = min(best, r.fun)
    assert abs(best / PESMIN_CH4CO2 - 1.0) < 1e-8


def test_rotor_dynamics_conserve_energy_and_reverse():
    sysd = oracle_system("ch4co2")
    p = oracle_params("ch4co2", 21, 200.0)
    qp, _ = O.sample(42, sysd, p, 200.0, 4)
    for q0 in qp:
        y, _ = O.propagate(sysd, p, q0, 4000.0)
        E0 = O.hamiltonian(sysd, q0)
        assert abs(O.hamiltonian(sysd, y) - E0) <= 1e-9 * max(abs(E0), 1e-3)
        yb = y.copy()
        yb[1::2] *= -1.0
        z, _ = O.propagate(sysd, p, yb, 4000.0)
        z[1::2] *= -1.0
        assert np.max(np.abs(np.cos(z) - np.cos(q0))[0::2]) < 1e-7


def test_sampler_layout_and_pair_state():
    sysd = oracle_system("ch4co2")
    p = oracle_params("ch4co2", 21, 200.0)
    qp, cand = O.sample(7, sysd, p, 300.0, 64)
    assert qp.shape == (64, 16) and cand >= 64
    assert np.all((qp[:, 4] >= 4.751) & (qp[:, 4] <= 40.0))
    assert np.all([O.hamiltonian(sysd, q) >= 0.0 for q in qp])
