"""The N2-Ar PIP-NN surfaces of the oracle, pinned against the reference.

- The PIP bases (and the PES basis' Jacobian) equal the reference's own generated
  basis functions, compiled where they lie under oracle/_ref.
- The PES network reproduces the reference's cached energy at infinite separation
  (en_inf, PES-IDS/ai_pes_n2_ar_pip_nn.cpp:130).
- The global minimum lies just above the example's pesmin of -97.3 cm^-1
  (examples/correlation_n2_ar.cpp:234), which bounds it for the rejection sampler.
- Analytic gradients match finite differences; the dipole's lab-frame form used by
  the kernels equals the reference's lab transform (examples/correlation_n2_ar.cpp:52-76).
"""
import numpy as np
import pytest

from oracle import oracle as O

HTOCM = 2.1947463136320e5
L_N2 = 2.07856749
EN_INF = 0.0384490895371528


def test_pip_bases_match_reference_sources():
    if not (O.ref_available() and __import__("os").path.exists(O.REF_DIR + "/libref_n2ar_pip.so")):
        pytest.skip("reference PIP bases not built")
    R = O.ref("n2ar_pip")
    rng = np.random.default_rng(0)
    for _ in range(100):
        y = rng.uniform(0.0, 1.0, 3)
        p, jac = O.n2ar_pes_pip(y)
        pr = np.zeros(17)
        jr = np.zeros(51)
        R.ref_n2ar_pes_pip(y, pr)
        R.ref_n2ar_pes_jac(y, jr)
        assert np.array_equal(p, pr)
        np.testing.assert_allclose(jac, jr.reshape(17, 3).T, rtol=0, atol=1e-14)
        y10 = rng.uniform(0.0, 1.0, 10)
        q = O.n2ar_dip_pip(y10)
        qr = np.zeros(308)
        R.ref_n2ar_dip_pip(y10, qr)
        assert np.array_equal(q, qr)


def test_energy_at_infinity_matches_reference_cache():
    for D in (1e4, 1e6):
        e, g = O.n2ar_energy_cm(np.array([L_N2, D, D]))
        assert abs(e - EN_INF) < 1e-10
        assert np.all(np.abs(g[1:]) < 1e-12)


def test_minimum_bounded_by_example_pesmin():
    sysd = O.System(O.SYS_N2AR, 1.0, 1.0)
    best = 0.0
    for R in np.linspace(6.0, 8.5, 51):
        for th in np.linspace(0.0, np.pi / 2, 46):
            best = min(best, O.pes(sysd, np.array([0.0, 0.0, R, 0.0, th])) * HTOCM)
    assert -97.3 <= best < -95.0


def test_gradient_matches_finite_differences():
    sysd = O.System(O.SYS_N2AR, 1.0, 1.0)
    rng = np.random.default_rng(1)
    for _ in range(40):
        q = np.array([rng.uniform(0, 2 * np.pi), np.arccos(rng.uniform(-1, 1)), rng.uniform(5.0, 14.0),
                      rng.uniform(0, 2 * np.pi), np.arccos(rng.uniform(-0.95, 0.95))])
        g = O.dpes(sysd, q)
        fd = np.zeros(5)
        for i in range(5):
            h = 1e-5
            qp, qm = q.copy(), q.copy()
            qp[i] += h
            qm[i] -= h
            fd[i] = (O.pes(sysd, qp) - O.pes(sysd, qm)) / (2 * h)
        assert np.max(np.abs(g - fd)) <= 1e-6 * np.max(np.abs(g)) + 1e-14


def test_dipole_lab_form_equals_reference_transform():
    sysd = O.System(O.SYS_N2AR, 1.0, 1.0)
    rng = np.random.default_rng(2)
    for _ in range(40):
        Phi, Th, R = rng.uniform(0, 2 * np.pi), np.arccos(rng.uniform(-1, 1)), rng.uniform(5.0, 30.0)
        ph, th = rng.uniform(0, 2 * np.pi), np.arccos(rng.uniform(-1, 1))
        rh = np.array([np.sin(Th) * np.cos(Phi), np.sin(Th) * np.sin(Phi), np.cos(Th)])
        u = np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
        x = rh @ u
        dm = O.n2ar_dip_mol(R, np.arccos(x))
        e = u - x * rh
        mu = dm[2] * rh + dm[0] * e / np.linalg.norm(e)
        d = O.dipole(sysd, np.array([Phi, Th, R, ph, th]))
        np.testing.assert_allclose(mu, d, rtol=1e-10, atol=1e-14)
        assert dm[1] == 0.0


def test_dipole_decays_with_distance():
    mags = [np.linalg.norm(O.n2ar_dip_mol(R, 0.7)) for R in (8.0, 12.0, 20.0, 40.0)]
    assert all(a > b for a, b in zip(mags, mags[1:]))
    assert mags[-1] < 1e-5
