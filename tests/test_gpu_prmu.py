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


@pytest.mark.parametrize("name,mode,even,odd", [("co2ar", 1, 0.0, 0.0), ("co2ar", 2, 1.0, 0.5),
                                                ("n2ar", 2, 0.0, 0.0)])
def test_requantized_spectrum_matches_oracle(name, mode, even, odd):
    """PR_MU with a LINEAR_MOLECULE_REQ_INTEGER / _HALFINTEGER monomer (src/trajectory.c:93-136,
    src/hawaii.c:3548-3662): the initial requantization, the torque-cache switch (5 samples,
    limit 1e-7 a.u.) that requantizes |j| at every sample while the pair is apart, and the
    half-integer spin weights, against the oracle's restatement in the reference's
    spherical coordinates.  Both land their steps on the sample times."""
    import hawaiihybrid_b200 as hh
    from tests.helpers import II_CO2, II_N2, MU_CO2AR, MU_N2AR
    N, dt, T, n, fmax, seed = 1024, 200.0, 300.0, 24, 500.0, 5
    t1 = hh.LINEAR_MOLECULE_REQ_INTEGER if mode == 1 else hh.LINEAR_MOLECULE_REQ_HALFINTEGER
    if name == "co2ar":
        ms = hh.init_ms(MU_CO2AR, t1, hh.ATOM, (II_CO2, II_CO2), None, seed)
    else:
        ms = hh.init_ms(MU_N2AR, t1, hh.ATOM, (II_N2, II_N2), None, seed, system_id=hh.SYSTEM_N2_AR)
    ms.torque_cache_len, ms.torque_limit = 5, 1e-7
    p = lib_params(name, N, dt)
    p.even_j_spin_weight, p.odd_j_spin_weight = even, odd
    nu, sf, cnt, _ = hh.prmu_iteration(ms, p, T, R0, n, fmax, False, 0, seed=seed)
    req = O.Req(mode, 5, 1e-7, even, odd)
    ref, cnt_ref = O.prmu_req(oracle_system(name), oracle_params(name, N, dt), T, R0, n, sf.size, seed, req)
    assert cnt == cnt_ref and cnt > 0
    assert np.max(np.abs(sf - ref)) <= 1e-6 * np.max(np.abs(ref))
    # requantization changes the spectrum against the plain monomer on the same draws
    ms_plain = lib_system(name, seed)
    _, sf0, _, _ = hh.prmu_iteration(ms_plain, lib_params(name, N, dt), T, R0, n, fmax, False, 0, seed=seed)
    assert np.max(np.abs(sf0 - sf)) > 1e-4 * np.max(np.abs(sf0))
