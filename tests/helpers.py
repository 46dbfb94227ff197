"""Shared fixtures: the benchmark workloads as oracle and library parameters."""
import numpy as np

from oracle import oracle as O

MU_HEAR = 6.632039160324215e+03
MU_CO2AR = 3.817083069753919e+04
II_CO2 = 2.819827114123505e+05
PESMIN_HEAR = -9.424412560638486e-05
PESMIN_CO2AR = -8.913727688689150e-04
# N2-Ar (constants.h:43-50,80,98; examples/correlation_n2_ar.cpp:214-234)
MU_N2AR = 30016.287464295514
II_N2 = 55141.90310147907
PESMIN_N2AR = -97.3 / 2.1947463136320e5
RMIN_N2AR = 4.51
# CH4-CO2 (example_configs/CF-F-CH4-CO2.conf:6,25,27-28,50,55)
MU_CH4CO2 = 2.141790360592430e+04
II_CH4 = 2.093840965876434e+04
PESMIN_CH4CO2 = -1.562522273622102e-03
RMIN_CH4CO2 = 4.751


def oracle_system(name):
    if name == "hear":
        return O.System(O.SYS_HEAR, MU_HEAR, 0.0)
    if name == "n2ar":
        return O.System(O.SYS_N2AR, MU_N2AR, II_N2)
    if name == "ch4co2":
        return O.System(O.SYS_CH4CO2, MU_CH4CO2, II_CO2, (II_CH4, II_CH4, II_CH4))
    return O.System(O.SYS_CO2AR, MU_CO2AR, II_CO2)


def _pesmin(name):
    return {"hear": PESMIN_HEAR, "co2ar": PESMIN_CO2AR, "n2ar": PESMIN_N2AR, "ch4co2": PESMIN_CH4CO2}[name]


def _rmin(name, Rmin):
    if Rmin is not None:
        return Rmin
    return {"n2ar": RMIN_N2AR, "ch4co2": RMIN_CH4CO2}.get(name, 4.0)


def oracle_params(name, N, dt, tol=1e-12, ps=O.PS_FREE_AND_METASTABLE, Rmin=None, Rmax=40.0, Rcut=40.0,
                  ppf=1.0):
    return O.Params(ps, _rmin(name, Rmin), Rmax, _pesmin(name), dt, N, Rcut, tol, tol, ppf, 50000)


def lib_params(name, N, dt, tol=1e-12, ps=1, Rmin=None, Rmax=40.0, Rcut=40.0, ppf=1.0, mixed_tol=1e-8):
    from hawaiihybrid_b200 import hawaii as H
    return H.CalcParams(ps=ps, sampler_Rmin=_rmin(name, Rmin), sampler_Rmax=Rmax, pesmin=_pesmin(name),
                        sampling_time=dt,
                        MaxTrajectoryLength=N, cvode_tolerance=tol, Rcut=Rcut,
                        partial_partition_function_ratio=ppf, mixed_tolerance=mixed_tol)


def lib_system(name, seed=1):
    import hawaiihybrid_b200 as hh
    if name == "hear":
        return hh.init_ms(MU_HEAR, hh.ATOM, hh.ATOM, None, None, seed)
    if name == "n2ar":
        return hh.init_ms(MU_N2AR, hh.LINEAR_MOLECULE, hh.ATOM, (II_N2, II_N2), None, seed,
                          system_id=hh.SYSTEM_N2_AR)
    if name == "ch4co2":
        return hh.init_ms(MU_CH4CO2, hh.ROTOR, hh.LINEAR_MOLECULE, (II_CH4, II_CH4, II_CH4), (II_CO2, II_CO2),
                          seed)
    return hh.init_ms(MU_CO2AR, hh.LINEAR_MOLECULE, hh.ATOM, (II_CO2, II_CO2), None, seed)


def rel_to_c0(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / abs(b[0]))
