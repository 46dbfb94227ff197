"""B200-native trajectory hot path of HAWAIIHYBRID (classical-trajectory CIA spectra).

The numerical work runs in libhh_cuda.so (hand-written sm_100a CUDA, C ABI in
include/hh_cuda.h); `hawaii` mirrors the reference's host interface on top of it.
"""
from . import _lib
from ._lib import HHError
from .hawaii import (ATOM, LINEAR_MOLECULE, LINEAR_MOLECULE_REQ_HALFINTEGER, LINEAR_MOLECULE_REQ_INTEGER, PAIR_STATE_ALL, PAIR_STATE_BOUND,
                     PAIR_STATE_FREE_AND_METASTABLE, PRECISION_FP64, PRECISION_MIXED, ROTOR,
                     SYSTEM_CH4_CO2, SYSTEM_CO2_AR, SYSTEM_HE_AR, SYSTEM_N2_AR, CalcParams, CFnc, CFncArray, MoleculeSystem,
                     SFnc, analytic_full_partition_function_by_V, calculate_correlation_and_save,
                     calculate_correlation_array_and_save, correlation_array_iteration,
                     calculate_m0, calculate_m0_vegas, calculate_m2, c_mpi_perform_integration, INTEGRAND_M0, INTEGRAND_PF, correlation_from_initial_conditions, correlation_iteration,
                     correlation_iterations, correlation_temperatures, prmu_iteration,
                     calculate_spectral_function_using_prmu_representation,
                     idct_cf_to_sf, init_ms, read_correlation_function, read_spectral_function,
                     sample_initial_conditions, write_correlation_function,
                     write_spectral_function)

__all__ = [n for n in dir() if not n.startswith("_")]
