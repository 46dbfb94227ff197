"""Algorithmic work model of the trajectory kernels (the roofline numerator).

Counts follow the usual convention: add, sub, mul = 1 flop, FMA = 2, divide,
square root and exp = 1 each.  Per-evaluation counts are static counts of the
formulas in csrc/hh_physics.cuh and csrc/hh_traj.cuh; the event counts (RHS
evaluations, steps, dense-output steps, samples) are measured by the kernels.
For the mixed path the work is split into the part done in FP32 (surfaces,
stage sums, dense-output increments) and the part done in FP64 (state
updates, tolerances, kinematic terms).
"""
from __future__ import annotations

# DOP853 tableau non-zeros (Hairer-Norsett-Wanner): stage rows 1..11, the
# solution row, the two error estimators, the three dense-output stages and
# the four dense-output rows
_STAGE_NNZ = (1, 2, 2, 3, 3, 4, 5, 6, 7, 8, 9)
_B_NNZ, _E5_NNZ, _E3_NNZ = 8, 8, 8
_EXTRA_NNZ = (8, 8, 8)
_D_NNZ = (12, 12, 12, 12)

# per-evaluation counts of the surfaces and equations of motion
SYSTEMS = {
    # He-Ar: |r|, V'(R) with 2 exp and the 6-term damped dispersion, force
    "hear": dict(n=6, nq=3, rhs=160, rhs_fp64_kin=3, dip=20),
    # CO2-Ar: |r|, |u|, x, Legendre P_l and P_l' to l = 10 (63), 6 radial cubics
    # with derivatives (72), 2 sums (24), force and torque (36), kinematics (15)
    "co2ar": dict(n=12, nq=6, rhs=234, rhs_fp64_kin=15, dip=196),
}


def per_event(system: str) -> dict:
    s = SYSTEMS[system]
    n, nq = s["n"], s["nq"]
    comb_sum = sum(2 * k for k in _STAGE_NNZ) * n + 2 * _B_NNZ * n          # stage sums
    comb_upd = 2 * (len(_STAGE_NNZ) + 1) * n                                 # y + h*acc
    err_sum = 2 * (_E5_NNZ + _E3_NNZ) * n
    err_fp64 = 8 * n + 20                                                    # scales, norm, controller
    dense_stage_sum = sum(2 * k for k in _EXTRA_NNZ) * n
    dense_stage_upd = 2 * len(_EXTRA_NNZ) * n
    dense_rows = nq * (7 + sum(2 * k + 1 for k in _D_NNZ))
    sample_interp = 14 * nq
    sample_fp64 = nq + 8                                                     # state add, |r|, Rcut test
    return dict(
        rhs=s["rhs"], rhs_fp64_kin=s["rhs_fp64_kin"], dip=s["dip"],
        step_sum=comb_sum + err_sum, step_fp64=comb_upd + err_fp64,
        dense_sum=dense_stage_sum + dense_rows, dense_fp64=dense_stage_upd,
        sample=sample_interp + s["dip"] + 6, sample_fp64=sample_fp64,
    )


def work(system: str, stats: dict, mixed: bool) -> dict:
    """FP32 and FP64 flops of one call from its measured event counts."""
    e = per_event(system)
    attempts = stats["n_steps"] + stats["n_rejected_steps"]
    n_rhs, n_dense, n_samp = stats["n_rhs"], stats["n_dense"], stats["n_samples"]
    phys = n_rhs * (e["rhs"] - e["rhs_fp64_kin"]) + n_samp * e["sample"] + attempts * e["step_sum"] \
        + n_dense * e["dense_sum"]
    f64 = n_rhs * e["rhs_fp64_kin"] + attempts * e["step_fp64"] + n_dense * e["dense_fp64"] \
        + n_samp * e["sample_fp64"]
    if mixed:
        return {"fp32": float(phys), "fp64": float(f64)}
    return {"fp32": 0.0, "fp64": float(phys + f64)}
