#!/usr/bin/env python3
"""Benchmark of the HAWAIIHYBRID trajectory hot path on B200.

Workload (one step): a CORRELATION_SINGLE pass over 102,400 CO2-Ar
trajectories at T = 300 K (Boltzmann-sampled initial conditions from the
MT19937 stream of seed 7, free+metastable pair state, R in [4, 40] bohr,
Rcut = 40 bohr), 32,768 dipole samples at dt = 100 a.u. forward and backward,
reduced into C(t).  The sampled initial conditions are generated on the
device, so the inputs are resident in HBM when a step starts.

  value   trajectories/s of the batched mixed-precision path (FP32 surfaces
          and stages, FP64 state and C(t)), whole job
  plain   the same for the FP64 drop-in path, same initial conditions
  e2e     the mixed path timed around the public call (hh_cuda_correlation via
          the Python mirror) with its host buffers

`python bench.py --impl reference` times the CPU restatement of the reference
path (oracle/, FP64, all host cores) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(system="co2ar", n_traj=102400, T=300.0, seed=7, N=32768, dt=100.0, Rmin=4.0, Rmax=40.0,
                Rcut=40.0, pesmin=-8.913727688689150e-04, mu=3.817083069753919e+04,
                II=2.819827114123505e+05, fp64_tol=1e-12)
# N2-Ar PIP-NN workload (rigid N2 + Ar, PES-IDS/ai_pes_n2_ar_pip_nn.cpp surfaces)
N2AR = dict(n_traj=262144, T=200.0, seed=7, N=16384, dt=100.0, Rmin=4.51, Rmax=40.0, Rcut=40.0,
            pesmin=-97.3 / 2.1947463136320e5, mu=30016.287464295514, II=55141.90310147907, fp64_tol=1e-12)
# CH4-CO2 rotor + linear molecule (example_configs/CF-F-CH4-CO2.conf: dt 200 a.u., 21 samples,
# R in [4.751, 40]); four temperature sets in one launch; stand-in PES, reference dipole
CH4CO2 = dict(n_per_T=262144, Ts=(100.0, 200.0, 300.0, 400.0), seed=2066497031, N=21, dt=200.0, Rmin=4.751,
              Rmax=40.0, Rcut=40.0, pesmin=-1.562522273622102e-03, mu=2.141790360592430e+04,
              II1=2.093840965876434e+04, II2=2.819827114123505e+05, fp64_tol=1e-12)
METRIC = "traj/s/GPU, batched mixed-precision vs FP64 plain, at C(t) rel err ≤1e-4"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
PROFILE_TRAFFIC = os.path.join(ROOT, "profiles", "traffic.json")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--trajectories", type=int, default=WORKLOAD["n_traj"])
    ap.add_argument("--samples", type=int, default=WORKLOAD["N"])
    ap.add_argument("--mixed-tol", type=float, default=3e-8)
    ap.add_argument("--plain-steps", type=int, default=2)
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample", type=int, default=4096)
    ap.add_argument("--no-n2ar", action="store_true", help="skip the N2-Ar PIP-NN workload")
    ap.add_argument("--n2ar-trajectories", type=int, default=N2AR["n_traj"])
    ap.add_argument("--no-ch4co2", action="store_true", help="skip the CH4-CO2 four-temperature workload")
    ap.add_argument("--ch4co2-per-T", type=int, default=CH4CO2["n_per_T"])
    ap.add_argument("--only-n2ar", action="store_true",
                    help="run only the N2-Ar workload and print its block as the JSON line")
    ap.add_argument("--only-ch4co2", action="store_true",
                    help="run only the CH4-CO2 workload and print its block as the JSON line")
    return ap.parse_args()


def bench_n2ar(args, hh, H):
    """N2-Ar PIP-NN: mixed (FP32 PES and stages, FP64 dipole and state) against the FP64
    path on the same initial conditions; two mixed iterations per launch."""
    w = N2AR
    n = args.n2ar_trajectories
    ms = hh.init_ms(w["mu"], hh.LINEAR_MOLECULE, hh.ATOM, (w["II"], w["II"]), None, w["seed"],
                    system_id=hh.SYSTEM_N2_AR)

    def params(tol=w["fp64_tol"]):
        return H.CalcParams(ps=hh.PAIR_STATE_FREE_AND_METASTABLE, sampler_Rmin=w["Rmin"], sampler_Rmax=w["Rmax"],
                            pesmin=w["pesmin"], sampling_time=w["dt"], MaxTrajectoryLength=w["N"],
                            cvode_tolerance=tol, Rcut=w["Rcut"], partial_partition_function_ratio=1.0,
                            mixed_tolerance=args.mixed_tol)

    c1, _, s1 = hh.correlation_iteration(ms, params(), w["T"], n, hh.PRECISION_MIXED, seed=w["seed"])
    hh.correlation_iterations(ms, params(), w["T"], n, 2, hh.PRECISION_MIXED, seed=w["seed"])  # buffers
    cs, _, sk = hh.correlation_iterations(ms, params(), w["T"], n, 2, hh.PRECISION_MIXED, seed=w["seed"])
    c64, _, s64 = hh.correlation_iteration(ms, params(), w["T"], n, hh.PRECISION_FP64, seed=w["seed"])
    mixed = 2 * n / (sk.as_dict()["total_ms"] / 1e3)
    plain = n / (s64.as_dict()["total_ms"] / 1e3)
    out = {"workload": f"N2-Ar PIP-NN, {n} trajectories x {w['N']} samples, dt {w['dt']} a.u., T {w['T']} K, "
                       f"R in [{w['Rmin']}, {w['Rmax']}]", "mixed_traj_per_s": mixed, "plain_fp64_traj_per_s": plain,
           "speedup_mixed_vs_plain": mixed / plain, "mixed_single_batch_traj_per_s": n / (s1.as_dict()["total_ms"] / 1e3),
           "mixed_rtol": args.mixed_tol, "fp64_rtol": w["fp64_tol"],
           "submission": "mixed: two iterations per launch; FP64: one iteration"}
    if not args.no_accuracy:
        c13, _, _ = hh.correlation_iteration(ms, params(1e-13), w["T"], n, hh.PRECISION_FP64, seed=w["seed"])
        c0 = abs(c64[0])
        d = np.abs(c1 - c64) / c0
        floor = np.abs(c13 - c64) / c0
        run = np.maximum.accumulate(floor)
        kh = int(np.argmax(run > 1e-8)) if np.any(run > 1e-8) else w["N"]
        kc = min(w["N"], int(1e5 / w["dt"]) + 1)
        out["accuracy"] = {"m0_rel_err": float(d[0]), "ct_err_t_le_1e5au": float(d[:kc].max()),
                           "fp64_horizon_k": kh, "ct_err_within_fp64_horizon": float(d[:max(kh, 1)].max()),
                           "ct_err_all": float(d.max()), "fp64_floor_all": float(floor.max())}
    return out


def bench_ch4co2(args, hh, H):
    """CH4-CO2: 4 x n_per_T trajectories (one set per temperature) in one call, mixed
    (FP32 PES, stages and batched dipole; FP64 state and C(t)) against the FP64 path on
    the same initial conditions."""
    w = CH4CO2
    n = args.ch4co2_per_T
    ms = hh.init_ms(w["mu"], hh.ROTOR, hh.LINEAR_MOLECULE, (w["II1"],) * 3, (w["II2"], w["II2"]), w["seed"])

    def params(tol=w["fp64_tol"]):
        return H.CalcParams(ps=hh.PAIR_STATE_FREE_AND_METASTABLE, sampler_Rmin=w["Rmin"], sampler_Rmax=w["Rmax"],
                            pesmin=w["pesmin"], sampling_time=w["dt"], MaxTrajectoryLength=w["N"],
                            cvode_tolerance=tol, Rcut=w["Rcut"], partial_partition_function_ratio=1.0,
                            mixed_tolerance=args.mixed_tol)

    def run(prec, tol=w["fp64_tol"]):
        return hh.correlation_temperatures(ms, params(tol), w["Ts"], n, prec, seed=w["seed"])

    run(hh.PRECISION_MIXED)   # grows the device buffers to the timed size
    cm, _, sm = run(hh.PRECISION_MIXED)
    run(hh.PRECISION_FP64)
    cp, _, sp = run(hh.PRECISION_FP64)
    tot = len(w["Ts"]) * n
    sm, sp = sm.as_dict(), sp.as_dict()
    mixed = tot / (sm["total_ms"] / 1e3)
    plain = tot / (sp["total_ms"] / 1e3)
    out = {"workload": f"CH4-CO2 rotor + linear molecule, {len(w['Ts'])} x {n} trajectories at T = "
                       f"{'/'.join(str(int(t)) for t in w['Ts'])} K in one call, {w['N']} samples at dt {w['dt']} a.u., "
                       f"R in [{w['Rmin']}, {w['Rmax']}]; stand-in site-site PES (the reference has no source for "
                       "its CH4-CO2 PES), reference dipole",
           "mixed_traj_per_s": mixed, "plain_fp64_traj_per_s": plain, "speedup_mixed_vs_plain": mixed / plain,
           "mixed_ms": sm["total_ms"], "plain_ms": sp["total_ms"], "mixed_rtol": args.mixed_tol,
           "fp64_rtol": w["fp64_tol"], "kernel_launches": sm["n_kernel_launches"],
           "stats_mixed": {k: sm[k] for k in ("n_candidates", "n_steps", "n_rhs", "n_samples", "n_failed",
                                              "sample_ms", "traj_ms")}}
    from hawaiihybrid_b200 import _lib
    s64, s32 = C.c_int(0), C.c_int(0)
    _lib.check(_lib.load().hh_cuda_debug_tuning(C.byref(s64), C.byref(s32)))
    out["dipole_records_per_lane"] = {"fp64": s64.value, "mixed": s32.value,
                                      "how": "timed per precision on the first call's records (the warm-up)"}
    if not args.no_accuracy:
        per_T = []
        for i in range(len(w["Ts"])):
            c0 = abs(cp[i][0])
            d = np.abs(cm[i] - cp[i]) / c0
            per_T.append({"T": w["Ts"][i], "m0_rel_err": float(d[0]), "ct_err_all": float(d.max())})
        out["accuracy"] = per_T
    return out


def config(args, ws):
    return {"workload": "CO2-Ar rigid linear rotor + atom, CORRELATION_SINGLE",
            "trajectories_per_gpu": args.trajectories, "temperature_K": WORKLOAD["T"],
            "seed": WORKLOAD["seed"], "samples": args.samples, "dt_au": WORKLOAD["dt"],
            "pair_state": "FREE_AND_METASTABLE", "R_range_bohr": [WORKLOAD["Rmin"], WORKLOAD["Rmax"]],
            "Rcut_bohr": WORKLOAD["Rcut"], "fp64_rtol": WORKLOAD["fp64_tol"], "mixed_rtol": args.mixed_tol,
            "parallelism": f"dp{ws}" if ws > 1 else "single-gpu",
            "l2": "256 MB flush before the timed call; working set (tables + C(t)) < 2 MB",
            "submission": "the K timed steps are one call of K iterations (hh_cuda_correlation_multi)"}


# ----------------------------------------------------------------------------
# reference arm: the CPU restatement of the reference path on all host cores
# ----------------------------------------------------------------------------
def run_reference(args, ws, rank):
    if rank != 0:
        return 0
    from oracle import oracle as O
    from tests.helpers import oracle_params, oracle_system
    cores = os.cpu_count() or 1
    sysd = oracle_system("co2ar")
    p = oracle_params("co2ar", args.samples, WORKLOAD["dt"], tol=WORKLOAD["fp64_tol"])
    S = args.cpu_sample
    qp, _ = O.sample(WORKLOAD["seed"], sysd, p, WORKLOAD["T"], S)
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        O.correlation_sum(sysd, p, qp, nthreads=cores)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
    ms = 1e3 * statistics.mean(times)
    v = S / (ms / 1e3)
    sample = (f"first {S} accepted trajectories of the workload (seed {WORKLOAD['seed']}), full "
              f"{args.samples}-sample correlation_eval each, FP64 DOP853 at rtol 1e-12, {cores} threads")
    line = {"metric": METRIC, "value": v, "unit": "traj/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (Boltzmann-sampled, MT19937 seed 7)",
            "config": config(args, 1), "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "traj/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "traj/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------
# clocks during the timed region
# ----------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.path = os.path.join("/tmp", f"hh_clocks_{os.getpid()}.csv")
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if not self.p:
            return None
        self.p.terminate()
        self.p.wait()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None
        reasons = set()
        for r in rows:
            for name, val in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"),
                                 r[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(rows)}


def main():
    args = parse()
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, ws, rank)

    import torch
    import hawaiihybrid_b200 as hh
    from hawaiihybrid_b200 import _lib, flops
    from hawaiihybrid_b200 import hawaii as H

    torch.cuda.set_device(local)
    if args.only_ch4co2:
        print(json.dumps({"ch4co2_four_temperatures": bench_ch4co2(args, hh, H)}), flush=True)
        return 0
    if args.only_n2ar:
        print(json.dumps({"n2ar_pip_nn": bench_n2ar(args, hh, H)}), flush=True)
        return 0
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    seed = WORKLOAD["seed"] + 1000 * rank   # one seed per rank, like the reference's per-rank seed table
    ms = hh.init_ms(WORKLOAD["mu"], hh.LINEAR_MOLECULE, hh.ATOM, (WORKLOAD["II"], WORKLOAD["II"]), None, seed,
                    device=local)
    n = args.trajectories

    def params(tol=WORKLOAD["fp64_tol"]):
        return H.CalcParams(ps=hh.PAIR_STATE_FREE_AND_METASTABLE, sampler_Rmin=WORKLOAD["Rmin"],
                            sampler_Rmax=WORKLOAD["Rmax"], pesmin=WORKLOAD["pesmin"],
                            sampling_time=WORKLOAD["dt"], MaxTrajectoryLength=args.samples,
                            cvode_tolerance=tol, Rcut=WORKLOAD["Rcut"], partial_partition_function_ratio=1.0,
                            mixed_tolerance=args.mixed_tol)

    p = params()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def run(prec, iters, pp=p):
        """`iters` consecutive iterations (steps) of n trajectories in one pipelined call."""
        flush.zero_()
        barrier()
        t0 = time.perf_counter()
        crlns, ntrajs, st = hh.correlation_iterations(ms, pp, WORKLOAD["T"], n, iters, prec, seed=seed)
        if dist:   # the one exchange step of the path: C(t) and ntraj summed over ranks
            t = torch.from_numpy(np.concatenate([crlns.ravel(), ntrajs])).to(f"cuda:{local}")
            dist.all_reduce(t)
            out = t.cpu().numpy()
            crlns = out[:crlns.size].reshape(crlns.shape)
            ntrajs = out[crlns.size:]
        wall = time.perf_counter() - t0
        barrier()
        return crlns, ntrajs, st.as_dict(), wall

    def max_over_ranks(x):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- mixed path: W single-step warm-ups (their latency is the single-batch figure) ----
    single_ms = []
    for _ in range(args.warmup):
        _, _, st_w, _ = run(hh.PRECISION_MIXED, 1)
        single_ms.append(st_w["total_ms"])
    single_mixed_ms = max_over_ranks(min(single_ms))
    # ---- K timed steps, submitted together so each step's long-lived trajectories
    # overlap the next step's bulk (C(t) kept per step).  One untimed call of the
    # same size first: it grows the library's device buffers to the timed size, so
    # no allocation falls inside the timed call ----
    clocks = Clocks(local)
    clocks.start()
    run(hh.PRECISION_MIXED, args.steps)
    crlns_m, _, last, wall_m = run(hh.PRECISION_MIXED, args.steps)
    ck = clocks.stop()
    launches = int(last["n_kernel_launches"])
    mixed_ms = max_over_ranks(last["total_ms"]) / args.steps
    mixed_wall = max_over_ranks(wall_m) / args.steps
    value = n * ws / (mixed_ms / 1e3)
    crln_m = crlns_m[0]

    # ---- plain FP64 path on the same initial conditions ----
    run(hh.PRECISION_FP64, max(1, args.plain_steps), params())  # warm-up at the timed size
    crlns_p, _, st_p, _ = run(hh.PRECISION_FP64, max(1, args.plain_steps))
    plain_ms = max_over_ranks(st_p["total_ms"]) / max(1, args.plain_steps)
    plain_value = n * ws / (plain_ms / 1e3)
    crln_p = crlns_p[0]

    # ---- accuracy of the mixed path against the FP64 path (same initial conditions) ----
    acc = None
    if not args.no_accuracy:
        c0 = abs(crln_p[0])
        d = np.abs(crln_m - crln_p) / c0
        kc = min(args.samples, int(1e5 / WORKLOAD["dt"]) + 1)   # collision window t <= 1e5 a.u.
        acc = {"m0_rel_err": float(abs(crln_m[0] - crln_p[0]) / c0),
               "ct_err_t_le_1e5au": float(d[:kc].max()),
               "ct_err_all": float(d.max())}
        # reproducibility of the FP64 answer itself: rtol 1e-13 against 1e-12
        crlns_t, _, _, _ = run(hh.PRECISION_FP64, 1, params(1e-13))
        floor = np.abs(crlns_t[0] - crln_p) / c0
        runmax = np.maximum.accumulate(floor)
        kh = int(np.argmax(runmax > 1e-8)) if np.any(runmax > 1e-8) else args.samples
        acc.update({"fp64_floor_all": float(floor.max()),
                    "fp64_horizon_k": kh, "fp64_horizon_t_au": kh * WORKLOAD["dt"],
                    "ct_err_within_fp64_horizon": float(d[:kh].max()) if kh > 0 else None,
                    "definition": "max_k |C_mixed - C_fp64| / C_fp64(0) on the first step's trajectories; "
                                  "fp64 horizon = first k where FP64 at rtol 1e-13 and 1e-12 differ by "
                                  "more than 1e-8 C(0)"})

    # ---- roofline of the trajectory kernel (mixed path) ----
    lib = _lib.load()
    p32, p64 = C.c_double(), C.c_double()
    _lib.check(lib.hh_cuda_fma_peak(_lib.HH_PRECISION_MIXED, C.byref(p32)))
    _lib.check(lib.hh_cuda_fma_peak(_lib.HH_PRECISION_FP64, C.byref(p64)))
    w = flops.work("co2ar", last, mixed=True)
    t_s = last["traj_ms"] / 1e3
    achieved = (w["fp32"] + w["fp64"]) / t_s / 1e12
    frac = (w["fp32"] / (p32.value * 1e12) + w["fp64"] / (p64.value * 1e12)) / t_s
    peak = achieved / frac if frac > 0 else None
    wp = flops.work("co2ar", st_p, mixed=False)
    frac_p = wp["fp64"] / (p64.value * 1e12) / (st_p["traj_ms"] / 1e3)
    # DRAM bytes per trajectory from one ncu capture of a single-iteration launch,
    # scaled to the timed launch's n * steps trajectories (initial conditions and
    # C(t) slices both grow with the trajectories a launch processes)
    traffic = None
    if os.path.exists(PROFILE_TRAFFIC):
        try:
            tr = json.load(open(PROFILE_TRAFFIC))
            traffic = tr["traj_kernel_mixed_bytes_per_trajectory"] * n * args.steps
        except (ValueError, OSError, KeyError, TypeError):
            traffic = None
    roof = {"bound": "fp32+fp64 CUDA-core FMA (no tensor or HBM bound: ~1e-3 B/flop)",
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": frac, "traffic": traffic,
            "kernel": "traj_kernel<CO2-Ar, float, float> (mixed)",
            "peak_source": f"measured in-process FMA loops: fp32 {p32.value:.1f}, fp64 {p64.value:.1f} TFLOP/s; "
                           "peak = the blend for this kernel's fp32/fp64 mix",
            "work_flops": w, "plain_fp64_frac": frac_p}

    # ---- CPU baseline: the oracle on a bounded sample (rank 0, one GPU) ----
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        from tests.helpers import oracle_params, oracle_system
        cores = os.cpu_count() or 1
        sysd = oracle_system("co2ar")
        op = oracle_params("co2ar", args.samples, WORKLOAD["dt"], tol=WORKLOAD["fp64_tol"])
        S = args.cpu_sample
        qp, _ = O.sample(WORKLOAD["seed"], sysd, op, WORKLOAD["T"], S)
        t0 = time.perf_counter()
        O.correlation_sum(sysd, op, qp, nthreads=cores)
        cs = time.perf_counter() - t0
        cpu = {"value": S / cs, "unit": "traj/s", "cores": cores, "kind": "port",
               "sample": f"first {S} accepted trajectories of the workload, FP64 DOP853 rtol 1e-12, "
                         f"{cores} threads, {cs:.1f} s"}

    n2ar = None
    if rank == 0 and ws == 1 and not args.no_n2ar:
        n2ar = bench_n2ar(args, hh, H)
    ch4co2 = None
    if rank == 0 and ws == 1 and not args.no_ch4co2:
        ch4co2 = bench_ch4co2(args, hh, H)

    if rank == 0:
        h2d = C.sizeof(_lib.CalcParamsC) + 8 + 4 + 8 + 4
        d2h = args.samples * 8 + 8 + C.sizeof(_lib.Stats)
        line = {"metric": METRIC, "value": value, "unit": "traj/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": mixed_ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "fp32 surfaces + fp64 state", "data": "synthetic (Boltzmann-sampled "
                "initial conditions, MT19937 seed 7 + 1000*rank)", "config": config(args, ws),
                "plain_fp64": {"value": plain_value, "unit": "traj/s", "ms_per_step": plain_ms,
                               "steps_per_call": max(1, args.plain_steps),
                               "mixed_steps_per_call": args.steps},
                "single_batch": {"mixed_traj_per_s": n * ws / (single_mixed_ms / 1e3),
                                 "mixed_ms": single_mixed_ms,
                                 "note": "one step submitted alone: its long-lived trajectories "
                                         "finish with the GPU mostly idle"},
                "speedup_mixed_vs_plain": value / plain_value,
                "accuracy": acc,
                "e2e": {"value": n * ws / mixed_wall, "unit": "traj/s", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h},
                "gpu_launches": launches, "clocks": ck, "roofline": roof, "cpu_baseline": cpu,
                "n2ar_pip_nn": n2ar,
                "ch4co2_four_temperatures": ch4co2,
                "stats_last_step": {k: last[k] for k in ("n_candidates", "n_steps", "n_rejected_steps", "n_rhs",
                                                         "n_samples", "n_dense", "n_failed", "sample_ms",
                                                         "traj_ms")}}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
