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
