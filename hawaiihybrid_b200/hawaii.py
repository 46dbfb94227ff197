"""Host-side mirror of HAWAIIHYBRID's trajectory-path interface over libhh_cuda.so.

Names, argument meaning and units follow the reference's C API
(src/hawaii.h): MonomerType / PairState values, CalcParams fields,
init_ms, calculate_correlation_and_save, idct_cf_to_sf, the CF/SF text
formats and analytic_full_partition_function_by_V.  Every numerical step runs
in the CUDA library; this module only marshals arguments, loops over
iterations and writes files.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math
import os
import time
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import HHError, check

# ---- constants (src/constants.h:8-53) ----
ALU = 5.29177210903e-11
Boltzmann = 1.380649e-23
Hartree = 4.3597447222071e-18
HTOCM = 2.1947463136320e5
HkT = Hartree / Boltzmann
ZeroCoeff = 0.00361479637 / (4.0 * math.pi)
SecondCoeff = 13856114.29344114
RAMTOAMU = 1822.888485332
m_He = 4.00260325413 * RAMTOAMU
m_Ar = 39.9623831237 * RAMTOAMU
m_C = 12.0 * RAMTOAMU
m_O = 15.994914619598 * RAMTOAMU
l_CO2 = 4.398
II_CO2 = m_O / 2.0 * l_CO2 * l_CO2

# ---- MonomerType (src/hawaii.h:183-190) ----
ATOM = 0
LINEAR_MOLECULE = 4
LINEAR_MOLECULE_REQ_INTEGER = 104
LINEAR_MOLECULE_REQ_HALFINTEGER = 204
ROTOR = 6

# ---- PairState (src/hawaii.h:290-300) ----
PAIR_STATE_NONE = 0
PAIR_STATE_FREE_AND_METASTABLE = 1
PAIR_STATE_BOUND = 2
PAIR_STATE_ALL = 3

# ---- surfaces available on the device ----
SYSTEM_HE_AR = _lib.HH_SYSTEM_HE_AR
SYSTEM_CO2_AR = _lib.HH_SYSTEM_CO2_AR
SYSTEM_N2_AR = _lib.HH_SYSTEM_N2_AR
SYSTEM_CH4_CO2 = _lib.HH_SYSTEM_CH4_CO2

PRECISION_FP64 = _lib.HH_PRECISION_FP64
PRECISION_MIXED = _lib.HH_PRECISION_MIXED


@dataclasses.dataclass
class CalcParams:
    """Subset of the reference's CalcParams (src/hawaii.h:313-365) used by the path."""
    ps: int = PAIR_STATE_FREE_AND_METASTABLE
    sampler_Rmin: float = 4.0
    sampler_Rmax: float = 40.0
    pesmin: float = 0.0
    sampling_time: float = 200.0
    MaxTrajectoryLength: int = 65536
    cvode_tolerance: float = 1e-12
    niterations: int = 1
    total_trajectories: int = 0
    cf_filename: Optional[str] = None
    Rcut: float = 40.0
    partial_partition_function_ratio: float = 0.0
    # CORRELATION_ARRAY (src/hawaii.h:313-365: num_satellite_temperatures, ...)
    satellite_temperatures: Sequence[float] = ()
    partial_partition_function_ratios: Sequence[float] = ()
    cf_filenames: Sequence[str] = ()
    # correlation_eval_zimmerman_trick instead of correlation_eval (BOUND pairs only)
    use_zimmermann_trick: bool = False
    # PR_MU spin weights of a LINEAR_MOLECULE_REQ_HALFINTEGER monomer (src/hawaii.h:336-337)
    even_j_spin_weight: float = 0.0
    odd_j_spin_weight: float = 0.0
    # device-path knobs (no reference counterpart)
    mixed_tolerance: float = 1e-8
    max_steps: int = 50000

    def to_c(self) -> _lib.CalcParamsC:
        return _lib.CalcParamsC(
            int(self.ps), float(self.sampler_Rmin), float(self.sampler_Rmax), float(self.pesmin),
            float(self.sampling_time), int(self.MaxTrajectoryLength), float(self.Rcut),
            float(self.cvode_tolerance), float(self.partial_partition_function_ratio),
            float(self.mixed_tolerance), int(self.max_steps), int(bool(self.use_zimmermann_trick)))


@dataclasses.dataclass
class MoleculeSystem:
    """The pair being simulated (src/hawaii.h:267-284) bound to a device surface."""
    system_id: int
    mu: float
    m1_type: int
    m2_type: int
    II1: tuple = (0.0, 0.0, 0.0)
    II2: tuple = (0.0, 0.0, 0.0)
    seed: int = 0
    device: int = 0
    # Monomer fields of a requantized monomer 1 (src/hawaii.h:210-235)
    torque_cache_len: int = 0
    torque_limit: float = 0.0

    @property
    def QP_SIZE(self) -> int:
        return 6 + (self.m1_type % 100) + (self.m2_type % 100)

    @property
    def Q_SIZE(self) -> int:
        return self.QP_SIZE // 2

    def desc(self) -> _lib.SystemDesc:
        # the device surfaces take the plain monomer types; requantization is set per call
        return _lib.SystemDesc(self.system_id, self.mu, self.m1_type % 100, self.m2_type % 100,
                               (C.c_double * 3)(*self.II1), (C.c_double * 3)(*self.II2))


def init_ms(mu: float, t1: int, t2: int, II1: Optional[Sequence[float]], II2: Optional[Sequence[float]],
            seed: int, system_id: Optional[int] = None, device: int = 0) -> MoleculeSystem:
    """init_ms (src/hawaii.c:173-270): bind the pair to the device and seed the sampler stream.

    system_id names the device surface (the role of the plugin .so in the reference);
    it defaults from the monomer types (ATOM+ATOM -> He-Ar, LINEAR+ATOM -> CO2-Ar,
    ROTOR+LINEAR -> CH4-CO2)."""
    if mu <= 0:
        raise ValueError(f"invalid reduced mass ({mu:.5e}) -- must be positive")
    if system_id is None:
        if t1 == ATOM and t2 == ATOM:
            system_id = SYSTEM_HE_AR
        elif t1 % 100 == LINEAR_MOLECULE and t2 == ATOM:
            system_id = SYSTEM_CO2_AR
        elif t1 == ROTOR and t2 == LINEAR_MOLECULE:
            system_id = SYSTEM_CH4_CO2
        else:
            raise HHError(_lib.HH_E_UNSUPPORTED_SYSTEM, "no device surface for these monomers")
    ms = MoleculeSystem(system_id, mu, t1, t2, tuple(II1 or (0, 0, 0)) + (0.0,) * (3 - len(II1 or (0, 0, 0))),
                        tuple(II2 or (0, 0, 0)) + (0.0,) * (3 - len(II2 or (0, 0, 0))), seed, device)
    L = _lib.load()
    check(L.hh_cuda_init(device, C.byref(ms.desc())))
    check(L.hh_cuda_seed(seed))
    return ms


@dataclasses.dataclass
class CFnc:
    t: np.ndarray
    data: np.ndarray
    ntraj: float = 0.0
    Temperature: float = 0.0
    normalized: bool = False

    @property
    def len(self) -> int:
        return int(self.data.size)


@dataclasses.dataclass
class SFnc:
    nu: np.ndarray
    data: np.ndarray
    ntraj: float = 0.0
    Temperature: float = 0.0
    normalized: bool = False

    @property
    def len(self) -> int:
        return int(self.data.size)


def _bind(ms: MoleculeSystem):
    L = _lib.load()
    check(L.hh_cuda_init(ms.device, C.byref(ms.desc())))
    return L


def sample_initial_conditions(ms: MoleculeSystem, params: CalcParams, Temperature: float, n: int,
                              seed: int = 0) -> tuple[np.ndarray, int]:
    """q_generator + p_generator + reject + pair-state filter for n accepted points."""
    L = _bind(ms)
    out = np.empty(n * ms.QP_SIZE, dtype=np.float64)
    nc = C.c_uint64()
    pc = params.to_c()
    check(L.hh_cuda_sample(C.byref(pc), Temperature, seed, n, out, C.byref(nc)))
    return out.reshape(n, ms.QP_SIZE), int(nc.value)


def correlation_iteration(ms: MoleculeSystem, params: CalcParams, Temperature: float, n: int,
                          precision: int = PRECISION_FP64, seed: int = 0):
    """One accumulation pass of calculate_correlation_and_save: returns
    (sum_i ppf * crln_i, n, stats)."""
    L = _bind(ms)
    crln = np.zeros(params.MaxTrajectoryLength, dtype=np.float64)
    ntraj = C.c_double()
    st = _lib.Stats()
    pc = params.to_c()
    check(L.hh_cuda_correlation(C.byref(pc), Temperature, seed, n, precision, crln,
                                C.byref(ntraj), C.byref(st)))
    return crln, ntraj.value, st


def correlation_iterations(ms: MoleculeSystem, params: CalcParams, Temperature: float, n_per_iteration: int,
                           n_iterations: int, precision: int = PRECISION_FP64, seed: int = 0):
    """n_iterations accumulation passes in one launch: returns
    (crln_sums[n_iterations, N], ntraj[n_iterations], stats)."""
    L = _bind(ms)
    crln = np.zeros(n_iterations * params.MaxTrajectoryLength, dtype=np.float64)
    ntraj = np.zeros(n_iterations, dtype=np.float64)
    st = _lib.Stats()
    pc = params.to_c()
    check(L.hh_cuda_correlation_multi(C.byref(pc), Temperature, seed, n_per_iteration, n_iterations,
                                      precision, crln, ntraj, C.byref(st)))
    return crln.reshape(n_iterations, -1), ntraj, st


def correlation_temperatures(ms: MoleculeSystem, params: CalcParams, temperatures: Sequence[float],
                             n_per_temperature: int, precision: int = PRECISION_FP64, seed: int = 0):
    """The CORRELATION_SINGLE pass at several temperatures in one launch: returns
    (crln_sums[nT, N], ntraj[nT], stats)."""
    L = _bind(ms)
    T = np.ascontiguousarray(temperatures, dtype=np.float64)
    crln = np.zeros(T.size * params.MaxTrajectoryLength, dtype=np.float64)
    ntraj = np.zeros(T.size, dtype=np.float64)
    st = _lib.Stats()
    pc = params.to_c()
    check(L.hh_cuda_correlation_temperatures(C.byref(pc), T, T.size, seed, n_per_temperature, precision,
                                             crln, ntraj, C.byref(st)))
    return crln.reshape(T.size, -1), ntraj, st


def prmu_iteration(ms: MoleculeSystem, params: CalcParams, Temperature: float, R0: float, n: int,
                   approximate_frequency_max: float, allow_truncating: bool = False,
                   precision: int = PRECISION_FP64, seed: int = 0):
    """One pass of calculate_spectral_function_using_prmu_representation_and_save
    (src/hawaii.c:3148-3978): returns (nu, sum over counted trajectories of
    SF_COEFF pR/mu sum_c |F_c|^2, counted trajectories, stats)."""
    L = _bind(ms)
    mode = {LINEAR_MOLECULE_REQ_INTEGER: _lib.HH_REQ_INTEGER,
            LINEAR_MOLECULE_REQ_HALFINTEGER: _lib.HH_REQ_HALFINTEGER}.get(ms.m1_type, _lib.HH_REQ_NONE)
    req = _lib.Requantization(mode, int(ms.torque_cache_len), float(ms.torque_limit),
                              float(params.even_j_spin_weight), float(params.odd_j_spin_weight))
    check(L.hh_cuda_set_requantization(C.byref(req)))
    N = int(params.MaxTrajectoryLength)
    cap = N // 2 + 2
    nu = np.zeros(cap)
    sf = np.zeros(cap)
    nf = C.c_size_t()
    ntraj = C.c_double()
    st = _lib.Stats()
    pc = params.to_c()
    try:
        check(L.hh_cuda_prmu(C.byref(pc), Temperature, R0, approximate_frequency_max, int(allow_truncating), seed,
                             n, precision, nu, sf, cap, C.byref(nf), C.byref(ntraj), C.byref(st)))
    finally:
        L.hh_cuda_set_requantization(None)
    k = nf.value
    return nu[:k], sf[:k], ntraj.value, st


def calculate_spectral_function_using_prmu_representation(ms: MoleculeSystem, params: CalcParams,
                                                           Temperature: float, R0: float,
                                                           approximate_frequency_max: float,
                                                           allow_truncating: bool = False,
                                                           precision: int = PRECISION_FP64) -> SFnc:
    """The PR_MU spectral function over params.niterations passes of
    params.total_trajectories / params.niterations trajectories, divided by the trajectories
    counted (src/hawaii.c:3974-3977)."""
    per = max(1, int(params.total_trajectories) // max(1, int(params.niterations)))
    total, nt, nu = None, 0.0, None
    for it in range(max(1, int(params.niterations))):
        nu, sf, c, _ = prmu_iteration(ms, params, Temperature, R0, per, approximate_frequency_max,
                                      allow_truncating, precision, seed=ms.seed if it == 0 else 0)
        total = sf if total is None else total + sf
        nt += c
    return SFnc(nu=nu, data=total / nt, ntraj=nt, Temperature=Temperature, normalized=True)


def correlation_from_initial_conditions(ms: MoleculeSystem, params: CalcParams, qp0: np.ndarray,
                                        precision: int = PRECISION_FP64):
    """correlation_eval + accumulation over caller-supplied phase points."""
    L = _bind(ms)
    qp0 = np.ascontiguousarray(qp0, dtype=np.float64).reshape(-1, ms.QP_SIZE)
    crln = np.zeros(params.MaxTrajectoryLength, dtype=np.float64)
    st = _lib.Stats()
    pc = params.to_c()
    check(L.hh_cuda_correlation_ic(C.byref(pc), qp0.ravel(), qp0.shape[0], precision, crln,
                                   C.byref(st)))
    return crln, st


def correlation_array_iteration(ms: MoleculeSystem, params: CalcParams, base_temperature: float, n: int,
                                precision: int = PRECISION_FP64, seed: int = 0):
    """One accumulation pass of calculate_correlation_array_and_save: returns
    (data[n_sat, N] = sum_i w_is * ratio_s * crln_i, nstar[n_sat], ntraj, stats)."""
    L = _bind(ms)
    Ts = np.ascontiguousarray(params.satellite_temperatures, dtype=np.float64)
    ratios = np.ascontiguousarray(params.partial_partition_function_ratios, dtype=np.float64)
    if Ts.size < 1 or ratios.size != Ts.size:
        raise ValueError("satellite_temperatures and partial_partition_function_ratios must have the same, "
                         "nonzero length")
    N = params.MaxTrajectoryLength
    data = np.zeros(Ts.size * N, dtype=np.float64)
    nstar = np.zeros(Ts.size, dtype=np.float64)
    ntraj = C.c_double()
    st = _lib.Stats()
    pc = params.to_c()
    check(L.hh_cuda_correlation_array(C.byref(pc), base_temperature, Ts, ratios, Ts.size, seed, n, precision,
                                      data, nstar, C.byref(ntraj), C.byref(st)))
    return data.reshape(Ts.size, N), nstar, ntraj.value, st


@dataclasses.dataclass
class CFncArray:
    """CFncArray (src/hawaii.h): one unnormalised C(t) per satellite temperature."""
    t: np.ndarray
    data: np.ndarray        # [n_sat, N]
    nstar: np.ndarray       # per satellite: sum of the trajectory weights
    ntraj: float
    satellite_temperatures: tuple


def calculate_correlation_array_and_save(ms: MoleculeSystem, params: CalcParams, base_temperature: float,
                                         precision: int = PRECISION_FP64, log=print) -> CFncArray:
    """calculate_correlation_array_and_save (src/hawaii.c:2361-2793): trajectories sampled
    at base_temperature, each added to the C(t) of every satellite temperature with the
    reference's Boltzmann reweighting; after every pass each satellite's CF file is
    rewritten, unnormalised, with ntraj = nstar (hawaii.c:2758-2771)."""
    if params.total_trajectories <= 0 or params.niterations < 1:
        raise ValueError("total_trajectories and niterations must be positive")
    if params.ps not in (PAIR_STATE_FREE_AND_METASTABLE, PAIR_STATE_BOUND):
        raise ValueError("CORRELATION_ARRAY supports the FREE_AND_METASTABLE and BOUND pair states")
    Ts = tuple(float(x) for x in params.satellite_temperatures)
    N = params.MaxTrajectoryLength
    total = CFncArray(t=np.linspace(0.0, params.sampling_time * (N - 1), N), data=np.zeros((len(Ts), N)),
                      nstar=np.zeros(len(Ts)), ntraj=0.0, satellite_temperatures=Ts)
    if params.cf_filenames and len(params.cf_filenames) != len(Ts):
        raise ValueError("one cf_filename per satellite temperature")
    per_iter = params.total_trajectories // params.niterations
    for it in range(params.niterations):
        data, nstar, ntraj, _ = correlation_array_iteration(ms, params, base_temperature, per_iter, precision)
        total.data += data
        total.nstar += nstar
        total.ntraj += ntraj
        if log:
            log(f"ITERATION {it + 1}/{params.niterations}: accumulated {int(total.ntraj)} trajectories. "
                "Saving the temporary results")
            for s, T in enumerate(Ts):
                if total.nstar[s] > 0:
                    m0 = total.data[s][0] / total.nstar[s] * ZeroCoeff / ALU ** 3
                    log(f"T = {T:.2f}: NSTAR = {total.nstar[s]:.2f}, M0 ESTIMATE FROM CF: {m0:.5e}")
        for s, fname in enumerate(params.cf_filenames):
            with open(fname, "w") as fp:
                write_correlation_function_ext(fp, CFnc(t=total.t, data=total.data[s], ntraj=total.nstar[s],
                                                        Temperature=Ts[s], normalized=False))
    return total


def calculate_correlation_and_save(ms: MoleculeSystem, params: CalcParams, Temperature: float,
                                   precision: int = PRECISION_FP64, log=print, group: int = 4) -> CFnc:
    """calculate_correlation_and_save (src/hawaii.c:2795-3119): niterations passes of
    total_trajectories/niterations trajectories, the CF file rewritten after each
    pass, the result normalised by ntraj."""
    if params.partial_partition_function_ratio <= 0:
        raise ValueError("partial_partition_function_ratio must be provided (> 0)")
    if params.total_trajectories <= 0 or params.niterations < 1:
        raise ValueError("total_trajectories and niterations must be positive")
    N = params.MaxTrajectoryLength
    total = CFnc(t=np.linspace(0.0, params.sampling_time * (N - 1), N), data=np.zeros(N),
                 ntraj=0.0, Temperature=Temperature, normalized=False)
    per_iter = params.total_trajectories // params.niterations
    fp = open(params.cf_filename, "w") if params.cf_filename else None
    try:
        it = 0
        while it < params.niterations:
            # a group of iterations shares one launch; the CF file is still
            # rewritten after every iteration, in order
            g = min(group, params.niterations - it)
            crlns, ntrajs, st = correlation_iterations(ms, params, Temperature, per_iter, g, precision)
            for j in range(g):
                total.data += crlns[j]
                total.ntraj += ntrajs[j]
                it += 1
                if log:
                    log(f"ITERATION {it}/{params.niterations}: accumulated {int(total.ntraj)} trajectories."
                        + (f" Saving the temporary result to '{params.cf_filename}'" if fp else ""))
                    m0 = total.data[0] / total.ntraj * ZeroCoeff / ALU ** 3
                    log(f"M0 ESTIMATE FROM CF: {m0:.5e}")
                if fp:
                    write_correlation_function_ext(fp, total)
    finally:
        if fp:
            fp.close()
    total.data = total.data / total.ntraj
    total.normalized = True
    return total


def idct_cf_to_sf(cf: CFnc) -> SFnc:
    """idct_cf_to_sf (src/hawaii.c:5569-5601).  Like the reference, the Connes
    apodization is applied to cf.data in place."""
    L = _lib.load()
    data = np.ascontiguousarray(cf.data, dtype=np.float64)
    if data is not cf.data:
        cf.data = data
    N = data.size
    dt = float(cf.t[1] - cf.t[0])
    nu = np.empty(N)
    sf = np.empty(N)
    check(L.hh_cuda_idct_cf_to_sf(data, N, dt, nu, sf))
    return SFnc(nu=nu, data=sf, ntraj=cf.ntraj, Temperature=cf.Temperature, normalized=cf.normalized)


def calculate_m0(ms: MoleculeSystem, params: CalcParams, temperatures: Sequence[float], n_samples: int,
                 seed: int = 1, precision: int = PRECISION_FP64) -> tuple[np.ndarray, np.ndarray]:
    """Zeroth moment M0(T) for every temperature from one batch of phase-space samples
    (the quantity the reference prints as "T = ... => M0", src/driver.c:3425-3431)."""
    L = _bind(ms)
    T = np.ascontiguousarray(temperatures, dtype=np.float64)
    m = np.empty(T.size)
    e = np.empty(T.size)
    pc = params.to_c()
    check(L.hh_cuda_m0(C.byref(pc), T, T.size, n_samples, seed, precision, m, e))
    return m, e


def calculate_m2(ms: MoleculeSystem, params: CalcParams, temperatures: Sequence[float], n_samples: int,
                 seed: int = 1) -> tuple[np.ndarray, np.ndarray]:
    """Second moment M2(T) for every temperature from one batch of phase-space samples,
    in FP64 (the quantity the reference prints as "T = ... => M2": calculate_M2,
    src/hawaii.c:1524-1617, and the VEGAS integrand_M2, src/hep_hawaii.cpp:228-330)."""
    L = _bind(ms)
    T = np.ascontiguousarray(temperatures, dtype=np.float64)
    m = np.empty(T.size)
    e = np.empty(T.size)
    pc = params.to_c()
    check(L.hh_cuda_m2(C.byref(pc), T, T.size, n_samples, seed, m, e))
    return m, e


def moment_sums(ms: MoleculeSystem, params: CalcParams, temperatures: Sequence[float], n_samples: int,
                sample_offset: int = 0, seed: int = 1, moment: int = 0,
                precision: int = PRECISION_FP64) -> tuple[np.ndarray, np.ndarray]:
    """Per-temperature sums (sum w, sum w^2) of the M0 (moment 0) or M2 (moment 2) integrand
    over the Philox samples [sample_offset, sample_offset + n_samples): one rank's share of
    mpi_calculate_M0 / mpi_calculate_M2 (src/hawaii.c:1620-1738, 1740-1856)."""
    L = _bind(ms)
    T = np.ascontiguousarray(temperatures, dtype=np.float64)
    sw = np.empty(T.size)
    sw2 = np.empty(T.size)
    pc = params.to_c()
    check(L.hh_cuda_moment_sums(C.byref(pc), T, T.size, n_samples, sample_offset, seed, moment, precision, sw, sw2))
    return sw, sw2


INTEGRAND_M0 = _lib.HH_INTEGRAND_M0
INTEGRAND_PF = _lib.HH_INTEGRAND_PF


def c_mpi_perform_integration(ms: MoleculeSystem, integrand: int, params: CalcParams, Temperature: float,
                              niterations: int, npoints: int, seed: int = 1) -> tuple[float, float]:
    """VEGAS integral of integrand_M0 / integrand_pf (src/hep_hawaii.cpp:122-201, 332-389):
    returns (m, q), the value and error before the driver's scaling."""
    L = _bind(ms)
    m, q = C.c_double(), C.c_double()
    pc = params.to_c()
    check(L.hh_cuda_vegas(C.byref(pc), int(integrand), float(Temperature), int(niterations), int(npoints),
                          int(seed), C.byref(m), C.byref(q)))
    return m.value, q.value


def calculate_m0_vegas(ms: MoleculeSystem, params: CalcParams, Temperature: float, niterations: int = 12,
                       npoints: int = 1000000, seed: int = 1) -> tuple[float, float]:
    """The CALCULATION_PHASE_SPACE_M0 case of the reference driver (src/driver.c:3390-3447):
    VEGAS M0 scaled by ZeroCoeff / analytic_full_partition_function_by_V; defaults
    hep_m0_niterations = 12, hep_m0_npoints = 1e6."""
    m, q = c_mpi_perform_integration(ms, INTEGRAND_M0, params, Temperature, niterations, npoints, seed)
    s = ZeroCoeff / analytic_full_partition_function_by_V(ms, Temperature)
    return m * s, q * s


def moment_scale(params: CalcParams, moment: int = 0) -> float:
    """M = moment_scale * <w>: ZeroCoeff (SecondCoeff) * 4 pi (Rmax - Rmin)."""
    coeff = ZeroCoeff if moment == 0 else SecondCoeff
    return coeff * 4.0 * math.pi * (params.sampler_Rmax - params.sampler_Rmin)


def moment_from_sums(sw: np.ndarray, sw2: np.ndarray, n_samples: int, scale: float) -> tuple[np.ndarray, np.ndarray]:
    """(M, one-sigma error) from the integrand sums over n_samples samples."""
    mean = np.asarray(sw) / n_samples
    var = np.maximum(np.asarray(sw2) / n_samples - mean * mean, 0.0)
    return scale * mean, scale * np.sqrt(var / n_samples)


def analytic_full_partition_function_by_V(ms: MoleculeSystem, Temperature: float) -> float:
    """src/hawaii.c:5071-5090 (ATOM-ATOM, LINEAR_MOLECULE-ATOM, ROTOR-LINEAR_MOLECULE)."""
    if ms.m1_type == ATOM and ms.m2_type == ATOM:
        return (2.0 * math.pi * ms.mu * Temperature / HkT) ** 1.5
    if ms.m1_type == LINEAR_MOLECULE and ms.m2_type == ATOM:
        return 4.0 * math.pi * (2.0 * math.pi * Temperature / HkT) ** 2.5 * ms.mu ** 1.5 * ms.II1[0]
    if ms.m1_type == ROTOR and ms.m2_type == LINEAR_MOLECULE:
        return (32.0 * math.pi ** 3 * (2.0 * math.pi * Temperature / HkT) ** 4.0 * ms.mu ** 1.5 *
                math.sqrt(ms.II1[0] * ms.II1[1] * ms.II1[2]) * ms.II2[0])
    raise NotImplementedError("analytic_full_partition_function_by_V")


# ---- CF / SF text files (src/hawaii.c:4150-4284, 4502-4597) ----
def _header(fp, kind: str, T: float, ntraj: float, n: int) -> None:
    fp.write("# HAWAII HYBRID v0.1\n")
    fp.write("# Saved on " + time.strftime("%Y-%m-%d %H:%M:%S") + "\n")
    fp.write(f"# TEMPERATURE: {T:.2f}\n")
    fp.write(f"# AVERAGE OVER {ntraj:.2f} TRAJECTORIES\n")
    fp.write(f"# {kind}: {n}\n")


def _write_native(fp, entry: str, x: np.ndarray, data: np.ndarray, T: float, ntraj: float,
                  normalized: bool) -> int:
    """Run one of the library's writers (hh_write_*_ext) on the open Python file fp."""
    if not normalized and ntraj <= 0:
        raise ValueError(f"cannot normalize: trajectories count is {ntraj:.2f}")
    fp.flush()
    libc = C.CDLL(None)
    libc.fdopen.restype = C.c_void_p
    libc.fdopen.argtypes = [C.c_int, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    cfp = libc.fdopen(os.dup(fp.fileno()), b"w")
    if not cfp:
        raise OSError("fdopen failed")
    try:
        fn = getattr(_lib.load(), entry)
        fn.restype = C.c_long
        fn.argtypes = [C.c_void_p, _lib._dp, _lib._dp, C.c_size_t, C.c_double, C.c_double, C.c_int]
        n = fn(cfp, np.ascontiguousarray(x, dtype=np.float64), np.ascontiguousarray(data, dtype=np.float64),
               len(data), float(T), float(ntraj), int(bool(normalized)))
    finally:
        libc.fclose(cfp)
    fp.seek(0, os.SEEK_END)
    if n < 0:
        raise HHError(int(n), "CF/SF writer failed")
    return int(n)


def write_correlation_function_ext(fp, cf: CFnc) -> int:
    """Rewrite an open CF file (truncate, write, flush, fsync): the library's
    hh_write_correlation_function_ext, the same bytes as the reference's writer."""
    return _write_native(fp, "hh_write_correlation_function_ext", cf.t, cf.data, cf.Temperature, cf.ntraj,
                         cf.normalized)


def write_correlation_function(filename: str, cf: CFnc) -> int:
    with open(filename, "w") as fp:
        return write_correlation_function_ext(fp, cf)


def write_spectral_function(filename: str, sf: SFnc) -> int:
    with open(filename, "w") as fp:
        return _write_native(fp, "hh_write_spectral_function_ext", sf.nu, sf.data, sf.Temperature, sf.ntraj,
                             sf.normalized)


def _read_table(filename: str):
    T = None
    ntraj = None
    rows = []
    with open(filename) as fh:
        for line in fh:
            if line.startswith("#"):
                if line.startswith("# TEMPERATURE:"):
                    T = float(line.split(":")[1])
                elif line.startswith("# AVERAGE OVER"):
                    ntraj = float(line.split()[3])
                continue
            if line.strip():
                a, b = line.split()
                rows.append((float(a), float(b)))
    if T is None or ntraj is None:
        raise ValueError(f"incomplete header in '{filename}'")
    arr = np.array(rows, dtype=np.float64).reshape(-1, 2)
    return T, ntraj, arr


def read_correlation_function(filename: str) -> CFnc:
    T, ntraj, a = _read_table(filename)
    return CFnc(t=a[:, 0].copy(), data=a[:, 1].copy(), ntraj=ntraj, Temperature=T, normalized=True)


def read_spectral_function(filename: str) -> SFnc:
    T, ntraj, a = _read_table(filename)
    return SFnc(nu=a[:, 0].copy(), data=a[:, 1].copy(), ntraj=ntraj, Temperature=T, normalized=True)
