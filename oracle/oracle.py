"""ctypes bindings to the CPU oracle (liboracle.so) and to the reference pieces
compiled under oracle/_ref.  TEST INFRASTRUCTURE ONLY: imported by tests/, the
smoke check and the CPU-baseline leg of bench.py, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

SYS_HEAR, SYS_CO2AR, SYS_N2AR, SYS_CH4CO2 = 0, 1, 2, 3
PS_FREE_AND_METASTABLE, PS_BOUND, PS_ALL = 1, 2, 3

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")


class System(C.Structure):
    _fields_ = [("system", C.c_int), ("mu", C.c_double), ("II", C.c_double), ("II1", C.c_double * 3)]


class Params(C.Structure):
    _fields_ = [
        ("pair_state", C.c_int),
        ("Rmin", C.c_double), ("Rmax", C.c_double), ("pesmin", C.c_double),
        ("sampling_time", C.c_double), ("N", C.c_size_t), ("Rcut", C.c_double),
        ("rtol", C.c_double), ("atol", C.c_double), ("ppf_ratio", C.c_double),
        ("max_steps", C.c_long), ("zimmermann", C.c_int),
    ]


class TrajStats(C.Structure):
    _fields_ = [
        ("nsteps", C.c_long), ("nrej", C.c_long), ("nrhs", C.c_long), ("nsamples", C.c_long),
        ("status_fwd", C.c_int), ("status_bwd", C.c_int), ("failed", C.c_int),
    ]


def build(ref: str | None = None) -> None:
    """Build liboracle.so and, when the reference checkout is present, oracle/_ref.

    `ref` (else the environment variable HH_REFERENCE_DIR) overrides the checkout
    location that oracle/Makefile reads the reference sources from."""
    ref = ref or os.environ.get("HH_REFERENCE_DIR")
    cmd = ["make", "-s", "-C", HERE] + ([f"REF={ref}"] if ref else []) + ["all"]
    subprocess.run(cmd, check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.hho_mt_stream.argtypes = [C.c_uint32, C.c_size_t, _u32p]
        L.hho_philox4x32_10.argtypes = [_u32p, _u32p, _u32p]
        for name in ("hho_hear_V", "hho_hear_dV", "hho_hear_dip"):
            getattr(L, name).restype = C.c_double
            getattr(L, name).argtypes = [C.c_double]
        L.hho_co2ar_V_mol.restype = C.c_double
        L.hho_co2ar_V_mol.argtypes = [C.c_double, C.c_double]
        L.hho_co2ar_dV_mol.argtypes = [C.c_double, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.hho_co2ar_dip_mol.argtypes = [C.c_double, C.c_double, _dp]
        L.hho_co2ar_lab_to_mol.argtypes = [_dp, _dp]
        L.hho_co2ar_jacobian.argtypes = [_dp, _dp]
        L.hho_pes.restype = C.c_double
        L.hho_pes.argtypes = [C.POINTER(System), _dp]
        L.hho_dpes.argtypes = [C.POINTER(System), _dp, _dp]
        L.hho_dipole.argtypes = [C.POINTER(System), _dp, _dp]
        L.hho_rhs.argtypes = [C.POINTER(System), _dp, _dp]
        L.hho_hamiltonian.restype = C.c_double
        L.hho_hamiltonian.argtypes = [C.POINTER(System), _dp]
        L.hho_qp_to_cart.argtypes = [C.POINTER(System), _dp, _dp]
        L.hho_sample.restype = C.c_long
        L.hho_sample.argtypes = [C.c_uint32, C.POINTER(System), C.POINTER(Params), C.c_double,
                                 C.c_size_t, _dp]
        L.hho_correlation_eval.argtypes = [C.POINTER(System), C.POINTER(Params), _dp, _dp,
                                           C.POINTER(TrajStats)]
        L.hho_correlation_parts.argtypes = [C.POINTER(System), C.POINTER(Params), _dp, _dp, _dp,
                                            C.POINTER(TrajStats)]
        L.hho_propagate.argtypes = [C.POINTER(System), C.POINTER(Params), _dp, C.c_double, _dp,
                                    C.POINTER(C.c_long)]
        L.hho_correlation_sum.argtypes = [C.POINTER(System), C.POINTER(Params), _dp, C.c_size_t,
                                          C.c_int, _dp, C.c_void_p]
        L.hho_idct_cf_to_sf.argtypes = [_dp, C.c_size_t, C.c_double, _dp, _dp]
        L.hho_m0.argtypes = [C.POINTER(System), C.POINTER(Params), _dp, C.c_int, C.c_uint64,
                             C.c_uint64, C.c_uint64, C.c_int, _dp, _dp]
        L.hho_m0_scale.restype = C.c_double
        L.hho_m0_scale.argtypes = [C.POINTER(Params)]
        L.hho_m2.argtypes = L.hho_m0.argtypes
        L.hho_m2_scale.restype = C.c_double
        L.hho_m2_scale.argtypes = [C.POINTER(Params)]
        L.hho_analytic_pf.restype = C.c_double
        L.hho_analytic_pf.argtypes = [C.POINTER(System), C.c_double]
        L.hho_n2ar_energy_cm.argtypes = [_dp, _dp]
        L.hho_n2ar_energy_cm.restype = C.c_double
        L.hho_n2ar_V_lab.argtypes = [_dp]
        L.hho_n2ar_V_lab.restype = C.c_double
        L.hho_n2ar_dip_mol.argtypes = [C.c_double, C.c_double, _dp]
        L.hho_n2ar_pes_pip.argtypes = [_dp, _dp, _dp]
        L.hho_n2ar_dip_pip.argtypes = [_dp, _dp]
        L.hho_array_weights.argtypes = [C.c_int, C.c_double, C.c_double, _dp, C.c_int, C.c_double, _dp]
        L.hho_correlation_sum_array.argtypes = [C.POINTER(System), C.POINTER(Params), _dp, C.c_size_t, C.c_int,
                                                _dp, C.c_int, _dp]
        L.hho_correlation_eval_zimmermann.argtypes = [C.POINTER(System), C.POINTER(Params), _dp, _dp,
                                                      C.POINTER(TrajStats)]
        L.hho_prmu.restype = C.c_long
        L.hho_prmu.argtypes = [C.POINTER(System), C.POINTER(Params), C.c_double, C.c_double, C.c_int, C.c_uint32,
                               C.c_size_t, _dp, C.c_size_t, C.c_void_p]
        L.hho_ch4co2_lab_to_kal.argtypes = [_dp, _dp]
        L.hho_ch4co2_dipole_kal.argtypes = [_dp, _dp]
        L.hho_ch4co2_V_lab.restype = C.c_double
        L.hho_ch4co2_V_lab.argtypes = [_dp]
        _lib = L
    return _lib


def qp_size(system: int) -> int:
    return {SYS_HEAR: 6, SYS_CH4CO2: 16}.get(system, 10)


def q_size(system: int) -> int:
    return qp_size(system) // 2


def mt_stream(seed: int, n: int) -> np.ndarray:
    out = np.empty(n, dtype=np.uint32)
    lib().hho_mt_stream(seed, n, out)
    return out


def philox(ctr, key) -> np.ndarray:
    out = np.empty(4, dtype=np.uint32)
    lib().hho_philox4x32_10(np.asarray(ctr, dtype=np.uint32), np.asarray(key, dtype=np.uint32), out)
    return out


def sample(seed, sysd, params, T, n):
    qp = np.empty(n * qp_size(sysd.system), dtype=np.float64)
    cand = lib().hho_sample(seed, C.byref(sysd), C.byref(params), T, n, qp)
    return qp.reshape(n, -1), cand


def correlation_eval(sysd, params, qp0):
    crln = np.zeros(params.N, dtype=np.float64)
    st = TrajStats()
    lib().hho_correlation_eval(C.byref(sysd), C.byref(params), np.ascontiguousarray(qp0, dtype=np.float64),
                               crln, C.byref(st))
    return crln, st


def correlation_eval_zimmermann(sysd, params, qp0):
    crln = np.zeros(params.N, dtype=np.float64)
    st = TrajStats()
    lib().hho_correlation_eval_zimmermann(C.byref(sysd), C.byref(params),
                                          np.ascontiguousarray(qp0, dtype=np.float64), crln, C.byref(st))
    return crln, st


def prmu(sysd, params, T, R0, n, L, seed, allow_trunc=False, with_qp=False):
    """PR_MU core: (unnormalised sf[0..L), trajectories counted[, drawn phase points])"""
    sf = np.zeros(L)
    qp = np.zeros((n, qp_size(sysd.system))) if with_qp else None
    cnt = lib().hho_prmu(C.byref(sysd), C.byref(params), T, R0, int(allow_trunc), seed, n, sf, L,
                         qp.ctypes.data_as(C.c_void_p) if with_qp else None)
    return (sf, cnt, qp) if with_qp else (sf, cnt)


class Req(C.Structure):
    _fields_ = [("mode", C.c_int), ("len", C.c_int), ("limit", C.c_double), ("even_w", C.c_double),
                ("odd_w", C.c_double)]


def prmu_req(sysd, params, T, R0, n, L, seed, req, allow_trunc=False):
    """PR_MU with requantization of the linear monomer: (unnormalised sf[0..L), counted)"""
    Lb = lib()
    Lb.hho_prmu_req.restype = C.c_long
    Lb.hho_prmu_req.argtypes = [C.POINTER(System), C.POINTER(Params), C.c_double, C.c_double, C.c_int, C.c_uint32,
                                C.c_size_t, C.POINTER(Req), _dp, C.c_size_t, C.c_void_p]
    sf = np.zeros(L)
    cnt = Lb.hho_prmu_req(C.byref(sysd), C.byref(params), T, R0, int(allow_trunc), seed, n, C.byref(req), sf, L,
                          None)
    return sf, cnt


def correlation_parts(sysd, params, qp0):
    fw = np.zeros(params.N)
    bw = np.zeros(params.N)
    st = TrajStats()
    lib().hho_correlation_parts(C.byref(sysd), C.byref(params), np.ascontiguousarray(qp0, dtype=np.float64),
                                fw, bw, C.byref(st))
    return fw, bw


def correlation_sum(sysd, params, qp0, nthreads=None, with_stats=False):
    qp0 = np.ascontiguousarray(qp0, dtype=np.float64)
    n = qp0.shape[0]
    out = np.zeros(params.N, dtype=np.float64)
    stats = (TrajStats * n)() if with_stats else None
    lib().hho_correlation_sum(C.byref(sysd), C.byref(params), qp0.ravel(), n,
                              nthreads or os.cpu_count(), out, stats)
    return (out, stats) if with_stats else out


def propagate(sysd, params, qp0, t_end):
    out = np.empty(qp_size(sysd.system), dtype=np.float64)
    ns = C.c_long()
    rc = lib().hho_propagate(C.byref(sysd), C.byref(params), np.ascontiguousarray(qp0, dtype=np.float64),
                             t_end, out, C.byref(ns))
    if rc:
        raise RuntimeError(f"oracle propagate failed: {rc}")
    return out, ns.value


def idct_cf_to_sf(cf, dt):
    cf = np.array(cf, dtype=np.float64)
    N = cf.size
    nu = np.empty(N)
    sf = np.empty(N)
    rc = lib().hho_idct_cf_to_sf(cf, N, dt, nu, sf)
    if rc:
        raise ValueError("length must be a power of two")
    return nu, sf, cf


def m0(sysd, params, T, n_samples, seed, offset=0, nthreads=None):
    T = np.ascontiguousarray(T, dtype=np.float64)
    ws = np.zeros(T.size)
    wq = np.zeros(T.size)
    lib().hho_m0(C.byref(sysd), C.byref(params), T, T.size, n_samples, seed, offset,
                 nthreads or os.cpu_count(), ws, wq)
    return ws, wq


def vegas(sysd, params, integrand, T, niter, npoints, seed, nthreads=None):
    """(m, q) of the VEGAS restatement (hho_vegas); integrand 0 = M0, 1 = partition function."""
    L = lib()
    L.hho_vegas.argtypes = [C.POINTER(System), C.POINTER(Params), C.c_int, C.c_double, C.c_uint64, C.c_uint64,
                            C.c_uint64, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    m, q = C.c_double(), C.c_double()
    rc = L.hho_vegas(C.byref(sysd), C.byref(params), int(integrand), float(T), int(niter), int(npoints), int(seed),
                     nthreads or os.cpu_count(), C.byref(m), C.byref(q))
    if rc:
        raise ValueError("unsupported system or arguments")
    return m.value, q.value


def analytic_pf(sysd, T):
    L = lib()
    L.hho_analytic_pf.restype = C.c_double
    L.hho_analytic_pf.argtypes = [C.POINTER(System), C.c_double]
    return L.hho_analytic_pf(C.byref(sysd), float(T))


def m0_scale(params):
    return lib().hho_m0_scale(C.byref(params))


def m2(sysd, params, T, n_samples, seed, offset=0, nthreads=None):
    T = np.ascontiguousarray(T, dtype=np.float64)
    ws = np.zeros(T.size)
    wq = np.zeros(T.size)
    lib().hho_m2(C.byref(sysd), C.byref(params), T, T.size, n_samples, seed, offset,
                 nthreads or os.cpu_count(), ws, wq)
    return ws, wq


def m2_scale(params):
    return lib().hho_m2_scale(C.byref(params))


def qp_to_cart(sysd, qp):
    qp = np.ascontiguousarray(qp, dtype=np.float64)
    out = np.empty({SYS_HEAR: 6, SYS_CH4CO2: 19}.get(sysd.system, 12))
    lib().hho_qp_to_cart(C.byref(sysd), qp, out)
    return out


def pes(sysd, q):
    return lib().hho_pes(C.byref(sysd), np.ascontiguousarray(q, dtype=np.float64))


def dpes(sysd, q):
    out = np.zeros(max(5, q_size(sysd.system)))
    lib().hho_dpes(C.byref(sysd), np.ascontiguousarray(q, dtype=np.float64), out)
    return out


def dipole(sysd, q):
    out = np.zeros(3)
    lib().hho_dipole(C.byref(sysd), np.ascontiguousarray(q, dtype=np.float64), out)
    return out


def rhs(sysd, y):
    y = np.ascontiguousarray(y, dtype=np.float64)
    out = np.zeros(y.size)
    lib().hho_rhs(C.byref(sysd), y, out)
    return out


def hamiltonian(sysd, qp):
    return lib().hho_hamiltonian(C.byref(sysd), np.ascontiguousarray(qp, dtype=np.float64))


def array_weights(pair_state, pesmin, T0, Ts, E):
    """CORRELATION_ARRAY reweighting of one trajectory of energy E (hawaii.c:2640-2664)."""
    Ts = np.ascontiguousarray(Ts, dtype=np.float64)
    w = np.zeros(Ts.size)
    lib().hho_array_weights(pair_state, pesmin, T0, Ts, Ts.size, E, w)
    return w


def correlation_sum_array(sysd, params, qp0, w, nthreads=None):
    """out[s] = sum_i w[i, s] * crln_i (w carries the partial partition function ratios)."""
    qp0 = np.ascontiguousarray(qp0, dtype=np.float64)
    w = np.ascontiguousarray(w, dtype=np.float64)
    n_sat = w.shape[1]
    out = np.zeros(n_sat * params.N)
    lib().hho_correlation_sum_array(C.byref(sysd), C.byref(params), qp0.ravel(), qp0.shape[0],
                                    nthreads or os.cpu_count(), w.ravel(), n_sat, out)
    return out.reshape(n_sat, params.N)


def ch4co2_lab_to_kal(q):
    out = np.zeros(5)
    lib().hho_ch4co2_lab_to_kal(np.ascontiguousarray(q, dtype=np.float64), out)
    return out


def ch4co2_dipole_kal(qkal):
    out = np.zeros(3)
    lib().hho_ch4co2_dipole_kal(np.ascontiguousarray(qkal, dtype=np.float64), out)
    return out


def n2ar_energy_cm(d):
    g = np.zeros(3)
    e = lib().hho_n2ar_energy_cm(np.ascontiguousarray(d, dtype=np.float64), g)
    return e, g


def n2ar_dip_mol(R, theta):
    out = np.zeros(3)
    lib().hho_n2ar_dip_mol(R, theta, out)
    return out


def n2ar_pes_pip(y):
    p = np.zeros(17)
    jac = np.zeros(51)
    lib().hho_n2ar_pes_pip(np.ascontiguousarray(y, dtype=np.float64), p, jac)
    return p, jac.reshape(3, 17)


def n2ar_dip_pip(y):
    p = np.zeros(308)
    lib().hho_n2ar_dip_pip(np.ascontiguousarray(y, dtype=np.float64), p)
    return p


# ---- reference pieces compiled from the reference sources (oracle/_ref) ----
_ref = {}


def ref_available() -> bool:
    return all(os.path.exists(os.path.join(REF_DIR, f)) for f in
               ("libref_mtwist.so", "libref_hear.so", "libref_co2ar_pes.so", "libref_co2ar_ids.so"))


def ref(name):
    if name not in _ref:
        L = C.CDLL(os.path.join(REF_DIR, f"libref_{name}.so"))
        if name == "mtwist":
            L.mt_seed32.argtypes = [C.c_uint32]
            L.mt_lrand.restype = C.c_uint32
            L.mt_drand.restype = C.c_double
        elif name == "hear":
            for f in ("V_HeAr", "dV_HeAr", "dip_HeAr"):
                getattr(L, f).restype = C.c_double
                getattr(L, f).argtypes = [C.c_double]
        elif name == "co2ar_pes":
            L.pes_init()
            L.pes_co2ar.restype = C.c_double
            L.pes_co2ar.argtypes = [C.c_double, C.c_double]
            L.dpes_co2ar.argtypes = [C.c_double, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        elif name == "co2ar_ids":
            L.ref_co2ar_dip_mol.argtypes = [C.c_double, C.c_double, _dp]
        elif name == "ch4co2_ids":
            for f in ("ref_ch4co2_dipole_vector", "ref_ch4co2_lab_to_kal", "ref_ch4co2_dipole_lab"):
                getattr(L, f).argtypes = [_dp, _dp]
            L.ref_ch4co2_init()
        elif name == "n2ar_pip":
            L.ref_n2ar_pes_pip.argtypes = [_dp, _dp]
            L.ref_n2ar_pes_jac.argtypes = [_dp, _dp]
            L.ref_n2ar_dip_pip.argtypes = [_dp, _dp]
        _ref[name] = L
    return _ref[name]
