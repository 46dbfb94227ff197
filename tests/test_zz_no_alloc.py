"""hh_cuda_m0_noalloc, the allocation-free M0 entry point, against hh_cuda_m0.

hh_cuda_m0_noalloc serves hosts that must not allocate device memory once their
run has started: a job sharing the GPU with an allocator that holds most of HBM
in its pool, where a mid-run cudaMalloc can fail, or a host overlapping M0 with
work on other streams, which a cudaFree would stall until the device drains.
Its block partials and results live in one fixed array inside the library.

Both entry points draw the same Philox samples and reduce them in the same
order, so the results agree to rounding; the test allows 1e-12 relative.  Each
case calls the allocation-free entry point twice in a row, so that the second
call runs on scratch left over from the first.  This file is named to run last,
after the other GPU tests have used the library; it also passes on its own in a
fresh process, where its first call is the one that looks up the scratch."""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import II_CO2, II_N2, MU_CO2AR, MU_HEAR, MU_N2AR, lib_params

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _init(name):
    from hawaiihybrid_b200 import _lib
    L = _lib.load()
    if name == "hear":
        d = _lib.SystemDesc(_lib.HH_SYSTEM_HE_AR, MU_HEAR, _lib.HH_MONOMER_ATOM, _lib.HH_MONOMER_ATOM)
    elif name == "n2ar":
        # the N2-Ar kernels stage the folded dipole models in dynamic shared memory
        d = _lib.SystemDesc(_lib.HH_SYSTEM_N2_AR, MU_N2AR, _lib.HH_MONOMER_LINEAR_MOLECULE,
                            _lib.HH_MONOMER_ATOM)
        d.II1[0] = d.II1[1] = II_N2
    else:
        d = _lib.SystemDesc(_lib.HH_SYSTEM_CO2_AR, MU_CO2AR, _lib.HH_MONOMER_LINEAR_MOLECULE,
                            _lib.HH_MONOMER_ATOM)
        d.II1[0] = d.II1[1] = II_CO2
    _lib.check(L.hh_cuda_init(0, C.byref(d)))
    return L, _lib


def _m0(L, entry, cp, T, n, seed, prec):
    m = np.zeros(T.size)
    e = np.zeros(T.size)
    rc = getattr(L, entry)(C.byref(cp), T, int(T.size), n, seed, prec, m, e)
    return rc, m, e


@pytest.mark.parametrize("name,prec", [("hear", 0), ("hear", 1), ("co2ar", 0), ("co2ar", 1),
                                       ("n2ar", 0), ("n2ar", 1)])
def test_noalloc_matches_m0(name, prec):
    L, _lib = _init(name)
    cp = lib_params(name, 64, 100.0).to_c()
    # 20 temperatures: one full chunk of 16 and a ragged one
    T = np.ascontiguousarray(np.linspace(100.0, 400.0, 20))
    n = 1 << 18
    rc, m_ref, e_ref = _m0(L, "hh_cuda_m0", cp, T, n, 4242, prec)
    assert rc == _lib.HH_OK
    for _ in range(2):
        rc, m, e = _m0(L, "hh_cuda_m0_noalloc", cp, T, n, 4242, prec)
        assert rc == _lib.HH_OK, L.hh_cuda_strerror(rc)
        np.testing.assert_allclose(m, m_ref, rtol=RTOL, atol=0)
        np.testing.assert_allclose(e, e_ref, rtol=RTOL, atol=0)
    assert np.all(m > 0)


def test_noalloc_rejects_too_many_temperatures():
    L, _lib = _init("hear")
    cp = lib_params("hear", 64, 100.0).to_c()
    T = np.full(_lib.HH_M0_NOALLOC_MAX_T + 1, 300.0)
    rc, m, _ = _m0(L, "hh_cuda_m0_noalloc", cp, T, 1024, 1, 0)
    assert rc == _lib.HH_E_SCRATCH_LIMIT
    assert b"HH_M0_NOALLOC_MAX_T" in L.hh_cuda_strerror(rc)
    assert np.all(m == 0)
    # the largest allowed request runs and matches hh_cuda_m0
    T = np.ascontiguousarray(np.linspace(50.0, 500.0, _lib.HH_M0_NOALLOC_MAX_T))
    rc, m_ref, _ = _m0(L, "hh_cuda_m0", cp, T, 1 << 16, 7, 0)
    assert rc == _lib.HH_OK
    rc, m, _ = _m0(L, "hh_cuda_m0_noalloc", cp, T, 1 << 16, 7, 0)
    assert rc == _lib.HH_OK
    np.testing.assert_allclose(m, m_ref, rtol=RTOL, atol=0)
