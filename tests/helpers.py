"""Shared fixtures: reference workloads as oracle and library parameters."""
import numpy as np

from oracle import oracle as O

MU_HEAR = 6.632039160324215e+03
MU_CO2AR = 3.817083069753919e+04
II_CO2 = 2.819827114123505e+05
PESMIN_HEAR = -9.424412560638486e-05
PESMIN_CO2AR = -8.913727688689150e-04


def oracle_system(name):
    if name == "hear":
        return O.System(O.SYS_HEAR, MU_HEAR, 0.0)
    return O.System(O.SYS_CO2AR, MU_CO2AR, II_CO2)


def oracle_params(name, N, dt, tol=1e-12, ps=O.PS_FREE_AND_METASTABLE, Rmin=4.0, Rmax=40.0, Rcut=40.0,
                  ppf=1.0):
    pesmin = PESMIN_HEAR if name == "hear" else PESMIN_CO2AR
    return O.Params(ps, Rmin, Rmax, pesmin, dt, N, Rcut, tol, tol, ppf, 50000)


def lib_params(name, N, dt, tol=1e-12, ps=1, Rmin=4.0, Rmax=40.0, Rcut=40.0, ppf=1.0, mixed_tol=1e-8):
    from hawaiihybrid_b200 import hawaii as H
    pesmin = PESMIN_HEAR if name == "hear" else PESMIN_CO2AR
    return H.CalcParams(ps=ps, sampler_Rmin=Rmin, sampler_Rmax=Rmax, pesmin=pesmin, sampling_time=dt,
                        MaxTrajectoryLength=N, cvode_tolerance=tol, Rcut=Rcut,
                        partial_partition_function_ratio=ppf, mixed_tolerance=mixed_tol)


def lib_system(name, seed=1):
    import hawaiihybrid_b200 as hh
    if name == "hear":
        return hh.init_ms(MU_HEAR, hh.ATOM, hh.ATOM, None, None, seed)
    return hh.init_ms(MU_CO2AR, hh.LINEAR_MOLECULE, hh.ATOM, (II_CO2, II_CO2), None, seed)


def rel_to_c0(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / abs(b[0]))
