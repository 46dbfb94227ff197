"""Algorithmic work model of the trajectory kernels (the roofline numerator).

Counts follow the usual convention: add, sub, mul = 1 flop, FMA = 2, divide,
square root and exp = 1 each.  Per-evaluation counts are static counts of the
formulas in csrc/hh_physics.cuh and csrc/hh_traj.cuh; the event counts (RHS
evaluations, steps, dense-output steps, samples) are measured by the kernels.
For the mixed path the work is split into the part done in FP32 (surfaces,
stage sums, dense-output increments) and the part done in FP64 (state
updates, error norm and step control, kinematic terms).
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
    # N2-Ar: two pair functions y(d) (exp, quintic switch, 25 each), the 17 PIPs and
    # their Jacobian over the monomial table (320), scaler (34), 32 hidden units x
    # (17 FMA forward + SiLU' with exp and divide (7) + 17 FMA backward) = 2400,
    # chain to d1, d2 (73), Cartesian forces and torques (70), kinematics (15).
    # Dipole: mixed path = FP32 Chebyshev cell (atan2, cell index, 2 x 10 x 10 FMA,
    # basis recurrences, rotation: 490); FP64 path = the folded network (2 ranges x
    # 34 x 40 FMA, 40 SiLU differences with expm1 and divide, outputs: 6500)
    "n2ar": dict(n=12, nq=6, rhs=2960, rhs_fp64_kin=15, dip=490, dip_fp64=6500),
}

# Monte Carlo moment integrand per sample (hh_m0.cuh), surface-precision part and the
# part in the accumulation precision (the compensated sum of w and the sum of w^2: 6
# operations per temperature, FP64 on the FP64 path, compensated FP32 on the mixed
# path).  CO2-Ar: angle transforms (30), surface value (Legendre recursion 40, six
# radial values 60, sums 12: 112), dipole sums (170), |mu|^2 (5), per temperature H,
# exp, weight (5 each).
M0_PER_SAMPLE = {"co2ar": dict(phys=30 + 112 + 170 + 5, per_T=5, per_T_acc=6)}

# CH4-CO2 batched dipole (ch4_dipole_kernel) per record: 4 FMA per (padded) entry
# of the coefficient stream (the per-power sums), Horner and Y1 product per group
# (5 per group end, about one per 4 entries), record geometry (quaternion matrix,
# two frame vectors, Y2 table of 91 values: about 600)
def ch4_dipole_flops(n_entries_padded: int, n_groups: int) -> int:
    return 8 * n_entries_padded + 10 * n_groups + 600


# CH4-CO2 tensor-core dipole (ch4_dipole_tc_kernel): per 128-record task, pass 0 runs two
# 208-column component tiles and pass 1 one, over K = 368 in chunks of 16, each MMA of
# M = 128, N = 208, K = 8 issued three times (A_hi B_hi, A_hi B_lo, A_lo B_hi)
CH4_TC_MMA_FLOPS_PER_TASK = 3 * 2 * 128 * (2 * 208 + 208) * 368


def ch4_tc_mma_flops(n_records: int) -> float:
    """MMA flops the tensor-core dipole kernel issues for n_records records (whole tasks of
    128; the per-piece padding of the last task is not counted)."""
    return float(n_records) / 128.0 * CH4_TC_MMA_FLOPS_PER_TASK


def per_event(system: str, mixed: bool = True) -> dict:
    s = dict(SYSTEMS[system])
    if not mixed and "dip_fp64" in s:
        s["dip"] = s["dip_fp64"]
    n, nq = s["n"], s["nq"]
    comb_sum = sum(2 * k for k in _STAGE_NNZ) * n + 2 * _B_NNZ * n          # stage sums
    comb_upd = 2 * (len(_STAGE_NNZ) + 1) * n                                 # y + h*acc
    err_sum = 2 * (_E5_NNZ + _E3_NNZ) * n                                  # error estimates (stage sums)
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


def m0_work(system: str, n_samples: int, nT: int, mixed: bool) -> dict:
    """FP32 and FP64 flops of one M0 call over n_samples samples and nT temperatures."""
    c = M0_PER_SAMPLE[system]
    phys = n_samples * (c["phys"] + nT * c["per_T"])
    acc = n_samples * nT * c["per_T_acc"]
    if mixed:
        return {"fp32": float(phys + acc), "fp64": 0.0}
    return {"fp32": 0.0, "fp64": float(phys + acc)}


def sample_work(system: str, stats: dict, mixed: bool) -> dict:
    """FP32 and FP64 flops of the per-sample work of one call (dense-output interpolation,
    dipole, product with mu0): the deferred sample kernels' share of `work`."""
    e = per_event(system, mixed)
    n_samp = stats["n_samples"]
    if mixed:
        return {"fp32": float(n_samp * e["sample"]), "fp64": float(n_samp * e["sample_fp64"])}
    return {"fp32": 0.0, "fp64": float(n_samp * (e["sample"] + e["sample_fp64"]))}


def work(system: str, stats: dict, mixed: bool) -> dict:
    """FP32 and FP64 flops of one call from its measured event counts."""
    e = per_event(system, mixed)
    attempts = stats["n_steps"] + stats["n_rejected_steps"]
    n_rhs, n_dense, n_samp = stats["n_rhs"], stats["n_dense"], stats["n_samples"]
    phys = n_rhs * (e["rhs"] - e["rhs_fp64_kin"]) + n_samp * e["sample"] + attempts * e["step_sum"] \
        + n_dense * e["dense_sum"]
    f64 = n_rhs * e["rhs_fp64_kin"] + attempts * e["step_fp64"] + n_dense * e["dense_fp64"] \
        + n_samp * e["sample_fp64"]
    if mixed:
        return {"fp32": float(phys), "fp64": float(f64)}
    return {"fp32": 0.0, "fp64": float(phys + f64)}
