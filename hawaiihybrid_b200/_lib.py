"""ctypes binding of libhh_cuda.so (C ABI declared in include/hh_cuda.h).

There is no CPU fallback: if the library is missing or no CUDA device is
visible, every call raises HHError.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libhh_cuda.so")

HH_OK = 0
HH_E_NOT_INITIALIZED = -1
HH_E_INVALID_ARGUMENT = -2
HH_E_CUDA = -3
HH_E_UNSUPPORTED_SYSTEM = -4
HH_E_OUT_OF_MEMORY = -5
HH_E_NOT_POWER_OF_TWO = -6
HH_E_SAMPLER = -7
HH_E_NO_DEVICE = -8
HH_E_SCRATCH_LIMIT = -9
HH_M0_NOALLOC_MAX_T = 256

HH_MONOMER_ATOM = 0
HH_MONOMER_LINEAR_MOLECULE = 4
HH_MONOMER_ROTOR = 6
HH_PAIR_STATE_FREE_AND_METASTABLE = 1
HH_PAIR_STATE_BOUND = 2
HH_PAIR_STATE_ALL = 3
HH_SYSTEM_HE_AR = 1
HH_SYSTEM_CO2_AR = 2
HH_SYSTEM_N2_AR = 3
HH_SYSTEM_CH4_CO2 = 4
HH_PRECISION_FP64 = 0
HH_PRECISION_MIXED = 1

# entry points declared in include/hh_cuda.h
EXPORTS = (
    "hh_cuda_init", "hh_cuda_seed", "hh_cuda_sample", "hh_cuda_correlation", "hh_cuda_correlation_multi",
    "hh_cuda_correlation_ic", "hh_cuda_m0", "hh_cuda_idct_cf_to_sf", "hh_cuda_strerror",
    "hh_cuda_mt_stream", "hh_cuda_debug_inject", "hh_cuda_debug_item_trace", "hh_cuda_fma_peak",
    "hh_cuda_shutdown", "hh_cuda_m0_noalloc", "hh_cuda_correlation_array", "hh_cuda_correlation_temperatures",
    "hh_cuda_prmu", "hh_cuda_debug_n2ar_dipole", "hh_cuda_m2", "hh_cuda_debug_tuning",
    "hh_cuda_debug_kernel_ms", "hh_cuda_debug_ch4co2_fold", "hh_cuda_moment_sums", "hh_cuda_debug_traj_tuning",
    "hh_cuda_debug_set_ch4_dipole", "hh_cuda_debug_set_defer", "hh_cuda_debug_set_defer_overlap", "hh_cuda_vegas",
    "hh_cuda_set_requantization",
    "hh_write_correlation_function_ext", "hh_write_spectral_function_ext",
)
HH_REQ_NONE, HH_REQ_INTEGER, HH_REQ_HALFINTEGER = 0, 1, 2
HH_INTEGRAND_M0 = 0
HH_INTEGRAND_PF = 1
# kernel classes of hh_cuda_debug_kernel_ms
HH_KT_NAMES = ("traj_bulk", "traj_solo", "ch4_dipole", "ch4_sort", "ch4_corr", "moment", "samples", "item_start")
HH_KT_COUNT = len(HH_KT_NAMES)


class HHError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (code {code})")
        self.code = code


class SystemDesc(C.Structure):
    _fields_ = [
        ("system_id", C.c_int), ("mu", C.c_double),
        ("monomer1_type", C.c_int), ("monomer2_type", C.c_int),
        ("II1", C.c_double * 3), ("II2", C.c_double * 3),
    ]


class Requantization(C.Structure):
    _fields_ = [("mode", C.c_int), ("torque_cache_len", C.c_size_t), ("torque_limit", C.c_double),
                ("even_j_spin_weight", C.c_double), ("odd_j_spin_weight", C.c_double)]


class CalcParamsC(C.Structure):
    _fields_ = [
        ("pair_state", C.c_int),
        ("sampler_Rmin", C.c_double), ("sampler_Rmax", C.c_double), ("pesmin", C.c_double),
        ("sampling_time", C.c_double), ("MaxTrajectoryLength", C.c_size_t), ("Rcut", C.c_double),
        ("cvode_tolerance", C.c_double), ("partial_partition_function_ratio", C.c_double),
        ("mixed_tolerance", C.c_double), ("max_steps", C.c_long), ("use_zimmermann_trick", C.c_int),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("n_candidates", C.c_uint64), ("n_accepted", C.c_uint64), ("n_steps", C.c_uint64),
        ("n_rejected_steps", C.c_uint64), ("n_rhs", C.c_uint64), ("n_samples", C.c_uint64),
        ("n_dense", C.c_uint64), ("n_failed", C.c_uint64), ("status", C.c_uint64 * 8),
        ("sample_ms", C.c_double), ("traj_ms", C.c_double), ("total_ms", C.c_double),
        ("n_kernel_launches", C.c_uint64),
    ]

    def as_dict(self) -> dict:
        d = {f: getattr(self, f) for f, _ in self._fields_ if f != "status"}
        d["status"] = list(self.status)[:6]
        return d


_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_lib = None


def load(path: str | None = None):
    """Load libhh_cuda.so; raises HHError when it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise HHError(HH_E_CUDA, f"CUDA library not built: {path} (run __graft_entry__.build())")
    L = C.CDLL(path)
    L.hh_cuda_init.argtypes = [C.c_int, C.POINTER(SystemDesc)]
    L.hh_cuda_seed.argtypes = [C.c_uint32]
    L.hh_cuda_sample.argtypes = [C.POINTER(CalcParamsC), C.c_double, C.c_uint32, C.c_uint64, _dp,
                                 C.POINTER(C.c_uint64)]
    L.hh_cuda_correlation.argtypes = [C.POINTER(CalcParamsC), C.c_double, C.c_uint32, C.c_uint64,
                                      C.c_int, _dp, C.POINTER(C.c_double), C.POINTER(Stats)]
    L.hh_cuda_correlation_multi.argtypes = [C.POINTER(CalcParamsC), C.c_double, C.c_uint32, C.c_uint64,
                                            C.c_uint32, C.c_int, _dp, _dp, C.POINTER(Stats)]
    L.hh_cuda_correlation_temperatures.argtypes = [C.POINTER(CalcParamsC), _dp, C.c_int, C.c_uint32, C.c_uint64,
                                                   C.c_int, _dp, _dp, C.POINTER(Stats)]
    L.hh_cuda_prmu.argtypes = [C.POINTER(CalcParamsC), C.c_double, C.c_double, C.c_double, C.c_int, C.c_uint32,
                               C.c_uint64, C.c_int, _dp, _dp, C.c_size_t, C.POINTER(C.c_size_t),
                               C.POINTER(C.c_double), C.POINTER(Stats)]
    L.hh_cuda_correlation_ic.argtypes = [C.POINTER(CalcParamsC), _dp, C.c_uint64, C.c_int, _dp,
                                         C.POINTER(Stats)]
    L.hh_cuda_m0.argtypes = [C.POINTER(CalcParamsC), _dp, C.c_int, C.c_uint64, C.c_uint64, C.c_int,
                             _dp, _dp]
    L.hh_cuda_m2.argtypes = [C.POINTER(CalcParamsC), _dp, C.c_int, C.c_uint64, C.c_uint64, _dp, _dp]
    L.hh_cuda_m0_noalloc.argtypes = L.hh_cuda_m0.argtypes
    L.hh_cuda_moment_sums.argtypes = [C.POINTER(CalcParamsC), _dp, C.c_int, C.c_uint64, C.c_uint64, C.c_uint64,
                                      C.c_int, C.c_int, _dp, _dp]
    L.hh_cuda_correlation_array.argtypes = [C.POINTER(CalcParamsC), C.c_double, _dp, _dp, C.c_int, C.c_uint32,
                                            C.c_uint64, C.c_int, _dp, _dp, C.POINTER(C.c_double),
                                            C.POINTER(Stats)]
    L.hh_cuda_idct_cf_to_sf.argtypes = [_dp, C.c_size_t, C.c_double, _dp, _dp]
    L.hh_cuda_strerror.restype = C.c_char_p
    L.hh_cuda_strerror.argtypes = [C.c_int]
    L.hh_cuda_mt_stream.argtypes = [C.c_uint32, C.c_uint64, _u32p]
    L.hh_cuda_debug_inject.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int]
    L.hh_cuda_debug_item_trace.argtypes = [C.c_void_p, C.c_uint64]
    L.hh_cuda_fma_peak.argtypes = [C.c_int, C.POINTER(C.c_double)]
    L.hh_cuda_debug_n2ar_dipole.argtypes = [C.c_int, _dp, _dp, C.c_uint64, _dp]
    L.hh_cuda_debug_tuning.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.hh_cuda_debug_kernel_ms.argtypes = [C.c_int, _dp, np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS"),
                                          C.c_int]
    L.hh_cuda_debug_ch4co2_fold.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.hh_cuda_debug_set_ch4_dipole.argtypes = [C.c_int, C.c_int]
    L.hh_cuda_debug_set_defer.argtypes = [C.c_int, C.POINTER(C.c_int)]
    L.hh_cuda_debug_set_defer_overlap.argtypes = [C.c_int, C.POINTER(C.c_int)]
    L.hh_cuda_set_requantization.argtypes = [C.POINTER(Requantization)]
    L.hh_cuda_vegas.argtypes = [C.POINTER(CalcParamsC), C.c_int, C.c_double, C.c_uint64, C.c_uint64, C.c_uint64,
                                C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.hh_cuda_debug_traj_tuning.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.hh_cuda_shutdown.restype = None
    for name in EXPORTS:
        if name not in ("hh_cuda_strerror", "hh_cuda_shutdown") and not name.startswith("hh_write_"):
            getattr(L, name).restype = C.c_int
    _lib = L
    return L


def check(code: int) -> None:
    if code != HH_OK:
        msg = load().hh_cuda_strerror(code).decode()
        raise HHError(code, msg)


def kernel_ms(enable: bool) -> dict:
    """Per-kernel-class device time accumulated since the last call (hh_cuda_debug_kernel_ms),
    then switch the timer on or off."""
    ms = np.zeros(HH_KT_COUNT)
    n = np.zeros(HH_KT_COUNT, dtype=np.uint64)
    check(load().hh_cuda_debug_kernel_ms(int(bool(enable)), ms, n, HH_KT_COUNT))
    return {name: {"ms": float(ms[i]), "launches": int(n[i])} for i, name in enumerate(HH_KT_NAMES)}


def ch4co2_fold_shape() -> tuple[int, int]:
    """(batches of 4 coefficient entries, groups) of the CH4-CO2 dipole stream per radial piece."""
    nb, ng = C.c_int(0), C.c_int(0)
    check(load().hh_cuda_debug_ch4co2_fold(C.byref(nb), C.byref(ng)))
    return nb.value, ng.value


def defer_samples(mode: int = -1) -> int:
    """Placement of the mixed path's sample dipoles (hh_cuda_debug_set_defer): 0 in the
    trajectory kernel, 1 CO2-Ar deferred to the sample kernels, 2 CO2-Ar and N2-Ar;
    -1 only reads it.  Returns the mode before the call."""
    prev = C.c_int(0)
    check(load().hh_cuda_debug_set_defer(int(mode), C.byref(prev)))
    return prev.value


def defer_overlap(on: int = -1) -> int:
    """Whether deferred samples of the bulk trajectory launch are evaluated beside the
    solo launch (hh_cuda_debug_set_defer_overlap): 1 yes, 0 after it, -1 only reads.
    Returns the setting before the call."""
    prev = C.c_int(0)
    check(load().hh_cuda_debug_set_defer_overlap(int(on), C.byref(prev)))
    return prev.value


def traj_tuning(precision: int, set_warps: int = 0, set_handoff_div: int = 0) -> tuple[int, int]:
    """(warps per block, hand-off divisor) of the trajectory launch for the bound system and
    precision (0, 0 before the autotuner ran); set_* > 0 fixes, < 0 forgets the pick."""
    w, d = C.c_int(0), C.c_int(0)
    check(load().hh_cuda_debug_traj_tuning(int(precision), int(set_warps), int(set_handoff_div),
                                           C.byref(w), C.byref(d)))
    return w.value, d.value
