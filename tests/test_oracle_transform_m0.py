"""CF->SF against the reference's golden pair and M0, M2 against the reference's
published physics values."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import oracle_params, oracle_system

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_idct_golden_pair():
    """tests/CF-F-He-Ar-1000.0.txt -> tests/SF-F-He-Ar-1000.0.txt (tests/convert-cf-to-sf.conf)."""
    g = np.load(os.path.join(GOLD, "cf_sf_he_ar_1000.npz"))
    nu, sf, cf_apod = O.idct_cf_to_sf(g["cf"], float(g["dt"]))
    peak = np.max(np.abs(g["sf"]))
    assert np.max(np.abs(sf - g["sf"])) / peak < 1e-6
    m = np.abs(g["sf"]) >= 1e-6 * peak
    assert np.max(np.abs(sf[m] - g["sf"][m]) / np.abs(g["sf"][m])) < 1e-6
    np.testing.assert_allclose(nu[::64][1:], g["sf_nu_every64"][1:], rtol=1e-9)
    # the reference apodizes its input in place
    N = g["cf"].size
    t = float(g["dt"]) * np.arange(N) / (float(g["dt"]) * N)
    np.testing.assert_allclose(cf_apod, g["cf"] * (1 - t * t) ** 2, rtol=1e-15)


def test_idct_rejects_non_power_of_two():
    with pytest.raises(ValueError):
        O.idct_cf_to_sf(np.ones(100), 1.0)


@pytest.mark.parametrize("name,T,Rmin,published,tol", [
    # example_configs/CF-F-CO2-Ar.conf.out:189 (VEGAS, 72 ranks): 6.25651e-04
    ("co2ar", 100.0, 4.0, 6.25651e-04, 0.01),
    # example_configs/CF-F-He-Ar.conf.out:190 (VEGAS): 2.08597e-06; CF-derived 2.10491e-06 (:12262)
    ("hear", 100.0, 3.0, 2.08597e-06, 0.015),
])
def test_m0_physics_anchor(name, T, Rmin, published, tol):
    p = oracle_params(name, 64, 100.0, Rmin=Rmin)
    n = 2_000_000
    ws, wq = O.m0(oracle_system(name), p, [T], n, 12345)
    m = O.m0_scale(p) * ws[0] / n
    err = O.m0_scale(p) * np.sqrt(wq[0] / n - (ws[0] / n) ** 2) / np.sqrt(n)
    assert abs(m - published) <= tol * published + 3 * err


@pytest.mark.parametrize("name,T,Rmin,published,tol", [
    # example_configs/CF-F-CO2-Ar.conf.out:238 (VEGAS, 72 ranks): 4.41296e-01 +- 0.08 %
    ("co2ar", 100.0, 4.0, 4.41296e-01, 0.01),
    # example_configs/CF-F-He-Ar.conf.out:239 (VEGAS): 1.34536e-02 +- 0.02 %
    ("hear", 100.0, 3.0, 1.34536e-02, 0.01),
])
def test_m2_physics_anchor(name, T, Rmin, published, tol):
    """The second moment on the M0 samples, with the momentum average of |dmu/dt|^2 taken
    at the sampled kinetic energy and dmu/dq by central differences in the reference's
    coordinates, against the reference's VEGAS values."""
    p = oracle_params(name, 64, 100.0, Rmin=Rmin)
    n = 2_000_000
    ws, wq = O.m2(oracle_system(name), p, [T], n, 12345)
    m = O.m2_scale(p) * ws[0] / n
    err = O.m2_scale(p) * np.sqrt(wq[0] / n - (ws[0] / n) ** 2) / np.sqrt(n)
    assert abs(m - published) <= tol * published + 3 * err


def test_oracle_vegas_reproduces_published_m0():
    """The oracle's VEGAS restatement of c_mpi_perform_integration(INTEGRAND_M0) (Lepage's
    grid refinement over the reference's transform_variables map), scaled like the driver
    by ZeroCoeff / pf_analytic, reproduces the published VEGAS M0 at 100 K, and its
    partition-function integral over the R shell matches the analytic value times the
    shell volume (1 % at 300 K, where the well adds a little)."""
    import math
    from hawaiihybrid_b200 import hawaii as H
    for name, published in (("co2ar", 6.25651e-4), ("hear", 2.08597e-6)):
        sysd, p = oracle_system(name), oracle_params(name, 64, 100.0)
        m, q = O.vegas(sysd, p, 0, 100.0, 12, 200_000, 1)
        pf = O.analytic_pf(sysd, 100.0)
        m0, e0 = m * H.ZeroCoeff / pf, q * H.ZeroCoeff / pf
        assert abs(m0 - published) <= 0.01 * published + 3 * e0
        mp, qp = O.vegas(sysd, p, 1, 300.0, 8, 100_000, 2)
        shell = 4.0 * math.pi / 3.0 * (p.Rmax ** 3 - p.Rmin ** 3)
        assert abs(mp / shell / O.analytic_pf(sysd, 300.0) - 1.0) < 0.01 + 3 * qp / mp
