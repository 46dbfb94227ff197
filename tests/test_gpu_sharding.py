"""Rank sharding of the moment integrals on the device: the integrand sums over
disjoint Philox counter ranges add up to the sums of one range covering them
(the partition the multi-GPU path uses, one range per rank), and a range that
starts at an offset matches the oracle's sums over the same samples."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import lib_params, lib_system, oracle_params, oracle_system

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,moment,prec", [("co2ar", 0, 0), ("co2ar", 0, 1), ("hear", 0, 0),
                                              ("n2ar", 0, 0), ("co2ar", 2, 0)])
def test_moment_sums_partition(name, moment, prec):
    import hawaiihybrid_b200 as hh
    from hawaiihybrid_b200 import hawaii as H
    ms = lib_system(name)
    p = lib_params(name, 64, 100.0)
    T = np.linspace(150.0, 400.0, 20)   # a full chunk of 16 temperatures and a ragged one
    n = 300_000
    sw, sw2 = H.moment_sums(ms, p, T, n, 0, seed=77, moment=moment, precision=prec)
    parts = [H.moment_sums(ms, p, T, n // 3, r * (n // 3), seed=77, moment=moment, precision=prec)
             for r in range(3)]
    # the mixed path sums a thread's samples in compensated FP32 (the block and launch
    # reductions are FP64), so another split of the samples over threads rounds
    # differently at the 1e-10 level; the FP64 path agrees to its own rounding
    rt = 1e-8 if prec == 1 else 1e-12
    np.testing.assert_allclose(sum(a for a, _ in parts), sw, rtol=rt)
    np.testing.assert_allclose(sum(b for _, b in parts), sw2, rtol=rt)
    # the moments of the whole range equal the library's own M0 / M2
    m, e = H.moment_from_sums(sw, sw2, n, H.moment_scale(p, moment))
    if moment == 0:
        m_lib, e_lib = hh.calculate_m0(ms, p, T, n, seed=77, precision=prec)
    else:
        m_lib, e_lib = hh.calculate_m2(ms, p, T, n, seed=77)
    np.testing.assert_allclose(m, m_lib, rtol=1e-14)
    np.testing.assert_allclose(e, e_lib, rtol=1e-12)


@pytest.mark.parametrize("moment", [0, 2])
def test_moment_sums_offset_matches_oracle(moment):
    from hawaiihybrid_b200 import hawaii as H
    ms = lib_system("co2ar")
    p = lib_params("co2ar", 64, 100.0)
    T = np.array([150.0, 250.0, 400.0])
    n, off = 100_000, 1_234_567
    sw, _ = H.moment_sums(ms, p, T, n, off, seed=5, moment=moment, precision=0)
    fn = O.m0 if moment == 0 else O.m2
    ws, _ = fn(oracle_system("co2ar"), oracle_params("co2ar", 64, 100.0), T, n, 5, offset=off)
    np.testing.assert_allclose(sw, ws, rtol=1e-10 if moment == 0 else 1e-5)
