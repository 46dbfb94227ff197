"""PR_MU spectral function (src/hawaii.c:3148-3978, without requantization) on the GPU
against the CPU oracle's restatement, through the C ABI: the same drawn phase points
(q_generator, R := R0, p_generator, inward pR), forward trajectories until R > R0, Connes
apodization, FFT and SF_COEFF pR/mu sum_c |F_c|^2."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import lib_params, lib_system, oracle_params, oracle_system

pytestmark = pytest.mark.gpu
R0 = 40.0


def _run(name, N, dt, T, n, fmax, seed, prec=0, trunc=False):
    import hawaiihybrid_b200 as hh
    ms = lib_system(name, seed)
    return hh.prmu_iteration(ms, lib_params(name, N, dt), T, R0, n, fmax, trunc, prec, seed=seed)


@pytest.mark.parametrize("name,dt,T,n", [("hear", 200.0, 300.0, 64), ("co2ar", 200.0, 300.0, 32),
                                         ("n2ar", 200.0, 300.0, 16)])
def test_fp64_spectrum_matches_oracle(name, dt, T, n):
    N, fmax, seed = 2048, 500.0, 42
    nu, sf, cnt, st = _run(name, N, dt, T, n, fmax, seed)
    ref, cnt_ref = O.prmu(oracle_system(name), oracle_params(name, N, dt), T, R0, n, sf.size, seed)
    assert cnt == cnt_ref
    assert np.max(np.abs(sf - ref)) <= 1e-8 * np.max(np.abs(ref))
    step = 1.0 / (dt * 2.4188843265857e-17) / 2.99792458e10 / N
    assert sf.size == int(fmax / step) + 1
    np.testing.assert_allclose(nu, step * np.arange(sf.size), rtol=1e-15)


def test_truncated_trajectories_are_skipped_or_kept():
    """N = 64 (12,800 a.u.): most trajectories are still inside R0 at the end."""
    name, N, dt, T, n, fmax, seed = "co2ar", 64, 200.0, 300.0, 48, 1000.0, 7
    _, sf0, c0, _ = _run(name, N, dt, T, n, fmax, seed, trunc=False)
    _, sf1, c1, _ = _run(name, N, dt, T, n, fmax, seed, trunc=True)
    r0, k0 = O.prmu(oracle_system(name), oracle_params(name, N, dt), T, R0, n, sf0.size, seed)
    r1, k1 = O.prmu(oracle_system(name), oracle_params(name, N, dt), T, R0, n, sf1.size, seed, allow_trunc=True)
    assert (c0, c1) == (k0, k1) and c1 == n and c0 < c1
    assert np.max(np.abs(sf1 - r1)) <= 1e-8 * np.max(np.abs(r1))
    if c0:
        assert np.max(np.abs(sf0 - r0)) <= 1e-8 * np.max(np.abs(r0))


def test_mixed_matches_fp64():
    name, N, dt, T, n, fmax, seed = "co2ar", 2048, 200.0, 300.0, 256, 500.0, 3
    _, s64, c64, _ = _run(name, N, dt, T, n, fmax, seed, prec=0)
    _, s32, c32, _ = _run(name, N, dt, T, n, fmax, seed, prec=1)
    assert c32 == c64
    assert np.max(np.abs(s32 - s64)) <= 1e-3 * np.max(np.abs(s64))


def test_rejects_unsupported():
    import hawaiihybrid_b200 as hh
    with pytest.raises(hh.HHError):   # N must be a power of two
        _run("hear", 1000, 200.0, 300.0, 4, 100.0, 1)
    with pytest.raises(hh.HHError):   # above the Nyquist frequency
        _run("hear", 1024, 200.0, 300.0, 4, 1e5, 1)
    ms = lib_system("ch4co2")
    with pytest.raises(hh.HHError):
        hh.prmu_iteration(ms, lib_params("ch4co2", 64, 200.0), 300.0, R0, 4, 100.0)
