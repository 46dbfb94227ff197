"""The C ABI library loads on a machine without a GPU, exports every entry point
declared in include/hh_cuda.h and fails cleanly without a device."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "hh_cuda.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(hh_cuda_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared()
    for n in ("hh_cuda_init", "hh_cuda_correlation", "hh_cuda_m0", "hh_cuda_idct_cf_to_sf",
              "hh_cuda_shutdown"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from hawaiihybrid_b200 import _lib
    L = _lib.load()
    for name in declared():
        assert hasattr(L, name), name
        assert name in _lib.EXPORTS


def test_struct_layouts_match_header():
    from hawaiihybrid_b200 import _lib
    assert C.sizeof(_lib.SystemDesc) == 4 + 4 + 8 + 4 + 4 + 48
    assert C.sizeof(_lib.CalcParamsC) == 8 + 8 * 4 + 8 + 8 * 4 + 8 + 8   # ... max_steps, use_zimmermann_trick
    assert C.sizeof(_lib.Stats) == 8 * 8 + 8 * 8 + 3 * 8 + 8


def test_errors_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("device present")
    from hawaiihybrid_b200 import _lib
    L = _lib.load()
    d = _lib.SystemDesc(1, 6632.0, 0, 0)
    assert L.hh_cuda_init(0, C.byref(d)) == _lib.HH_E_NO_DEVICE
    assert L.hh_cuda_seed(1) == _lib.HH_E_NOT_INITIALIZED
    assert b"no CUDA device" in L.hh_cuda_strerror(_lib.HH_E_NO_DEVICE)
    import hawaiihybrid_b200 as hh
    with pytest.raises(hh.HHError):
        hh.init_ms(6632.0, hh.ATOM, hh.ATOM, None, None, 1)


def test_no_cpu_fallback_in_product():
    """The product package never imports the oracle."""
    pkg = os.path.join(ROOT, "hawaiihybrid_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith(".py"):
                src = open(os.path.join(dirpath, f)).read()
                assert not re.search(r"^\s*(from|import)\s+oracle", src, flags=re.M), f
