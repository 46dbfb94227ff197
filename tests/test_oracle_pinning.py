"""The CPU oracle against the reference's own code (golden fixtures generated from
the reference sources compiled in oracle/_ref, tests/golden/make_golden.py) and
against the reference's known answers."""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def g():
    return np.load(os.path.join(GOLD, "ref_surfaces.npz"))


def test_mt19937_matches_mtwist(g):
    for seed in (42, 7, 1):
        assert np.array_equal(O.mt_stream(seed, 4000), g[f"mt{seed}"])


def test_mt19937_seed42_first_draws():
    # mt_seed32(42); mt_drand() x3 with the reference's mtwist
    d = O.mt_stream(42, 3).astype(np.float64) * 2.0 ** -32
    assert d.tolist() == [0.5133931515738368, 0.7469599430914968, 0.13660536729730666]


def test_philox_known_answers():
    # Random123 philox4x32-10 known-answer vectors
    assert O.philox([0, 0, 0, 0], [0, 0]).tolist() == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert O.philox([0xffffffff] * 4, [0xffffffff] * 2).tolist() == [0x408f276d, 0x41c83b0e, 0xa20bc7c6,
                                                                      0x6d5451fd]
    assert O.philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344],
                    [0xa4093822, 0x299f31d0]).tolist() == [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_hear_surfaces(g):
    L = O.lib()
    R = g["hear_R"]
    ref = g["hear"]
    got = np.array([[L.hho_hear_V(r), L.hho_hear_dV(r), L.hho_hear_dip(r)] for r in R])
    for j in range(3):
        scale = np.max(np.abs(ref[:, j]))
        assert np.max(np.abs(got[:, j] - ref[:, j])) <= 1e-11 * scale


def test_hear_pesmin_known_answer():
    # pesmin of example_configs/CF-F-He-Ar.conf is V_HeAr at its minimum
    assert abs(O.lib().hho_hear_V(6.597835932201344) / -9.424412560638486e-05 - 1.0) < 1e-13


def test_co2ar_surfaces(g):
    L = O.lib()
    R, Th, ref = g["co2ar_R"], g["co2ar_theta"], g["co2ar"]
    got = []
    for r, t in zip(R, Th):
        a, b = C.c_double(), C.c_double()
        L.hho_co2ar_dV_mol(r, t, a, b)
        d = np.zeros(3)
        L.hho_co2ar_dip_mol(r, t, d)
        got.append([L.hho_co2ar_V_mol(r, t), a.value, b.value, d[0], d[2]])
    got = np.array(got)
    # errors measured against the largest magnitude in each R band: the
    # reference's monomial splines cancel near zeros of each function
    for lo, hi in ((3.5, 4.5), (4.5, 10.0), (10.0, 20.0), (20.0, 30.0), (30.0, 46.0)):
        m = (R >= lo) & (R < hi)
        for j in range(5):
            scale = np.max(np.abs(ref[m, j]))
            assert np.max(np.abs(got[m, j] - ref[m, j])) <= 1e-10 * scale, (lo, hi, j)


def test_co2ar_minimum_known_answer():
    # PES-IDS/ai_pes_co2ar.h:25-27: V(6.4966051519, pi/2) = -195.6337098547 cm^-1
    v = O.lib().hho_co2ar_V_mol(6.4966051519, np.pi / 2) * 2.1947463136320e5
    assert abs(v - (-195.6337098547)) < 1e-8


def test_jacobian_against_finite_differences():
    """examples/trajectory_co2_ar.cpp:64-113: analytic frame Jacobian vs 6th-order FD at
    qlab = {0.1, 0.2, 5.0, 0.3, 0.4}, tolerance 1e-9."""
    L = O.lib()
    q = np.array([0.1, 0.2, 5.0, 0.3, 0.4])
    jac = np.zeros(25)
    L.hho_co2ar_jacobian(q, jac)
    jac = jac.reshape(5, 5)

    def tomol(x):
        o = np.zeros(5)
        L.hho_co2ar_lab_to_mol(np.ascontiguousarray(x), o)
        return o
    h = 1e-3
    coef = {-3: -1 / 60, -2: 3 / 20, -1: -3 / 4, 1: 3 / 4, 2: -3 / 20, 3: 1 / 60}
    num = np.zeros((5, 5))
    for i in range(5):
        acc = np.zeros(5)
        for k, c in coef.items():
            x = q.copy()
            x[i] += k * h
            acc += c * tomol(x)
        num[i] = acc / h
    np.testing.assert_allclose(jac, num, atol=1e-9, rtol=0)


@pytest.mark.parametrize("name,qp", [
    # examples/correlation_he_ar.cpp:69-76
    ("hear", [1.748408280024098e-01, 8.000086892719947e+00, 2.043243374007463e-01,
              1.292311668112794e+01, 2.966821669009366e+01, -3.786729452372973e-00]),
    # examples/trajectory_co2_ar.cpp:133-144
    ("co2ar", [1.748408280024098e-01, 8.000086892719947e+00, 2.043243374007463e-01,
               1.292311668112794e+01, 19.066821669009366e+00, -0.186729452372973e-01,
               1.462013919064840e+00, 0.199991310728005e+01, 1.700437238862704e+00,
               0.160851788770303e+01]),
])
def test_rhs_against_numerical_hamiltonian_derivatives(name, qp):
    """Hamilton's equations vs 6th-order FD of the Hamiltonian, tolerance 1e-4
    (the reference's test_rhs)."""
    from tests.helpers import oracle_system
    L = O.lib()
    sysd = oracle_system(name)
    qp = np.array(qp)
    n = qp.size
    yd = np.zeros(n)
    L.hho_rhs(C.byref(sysd), qp, yd)
    h = 1e-3
    coef = {-3: -1 / 60, -2: 3 / 20, -1: -3 / 4, 1: 3 / 4, 2: -3 / 20, 3: 1 / 60}
    num = np.zeros(n)
    for i in range(n):
        acc = 0.0
        for k, c in coef.items():
            x = qp.copy()
            x[i] += k * h
            acc += c * L.hho_hamiltonian(C.byref(sysd), np.ascontiguousarray(x))
        dH = acc / h
        # dq/dt = dH/dp, dp/dt = -dH/dq
        if i % 2 == 0:
            num[i + 1] = -dH
        else:
            num[i - 1] = dH
    for i in range(n):
        assert abs(yd[i] - num[i]) <= 1e-4 * max(1.0, abs(num[i])), (i, yd[i], num[i])
