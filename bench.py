#!/usr/bin/env python
"""Descent-step throughput of the constrained fractional-Sobolev step on B200.

Workload (the reference's precision-form configuration): a seeded random-walk
closed knot with V = E = 8192 (3-D Gaussian steps of sigma 1/sqrt(V), closed by
drift removal, total length 10), tangent-point alpha=3, beta=6, eps=1e-10,
constraint set [barycenter, totalLength] frozen at the initial curve, frozen
projection (the app's default), analytical dE. One step = one sobolevStepSet
(gradient, Gram assembly, structured saddle solve, Armijo line search with
back-projection) from the same input curve.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl repulsive|reference]

Multi-GPU: replicas only (every rank runs its own curve, no collective on the
data path); value = steps of all ranks / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "descent steps/s at V=8192: mixed+batched vs plain FP64 GPU, at <=1e-8 rel energy err"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="repulsive", choices=["repulsive", "reference"])
    p.add_argument("--V", type=int, default=8192)
    p.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of oracle work")
    return p.parse_args()


def workload(V):
    from repulsive_test2_b200 import api as T
    from repulsive_test2_b200 import fixtures as F

    v, e = F.random_walk_knot(V, seed=1)
    blocks = [T.barycenterBlock(T.barycenterTarget(v, e)), T.totalLengthBlock(T.totalLength(v, e))]
    return v, e, blocks


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


def fp64_gemm_peak(torch, dev):
    """cuBLAS FP64 GEMM rate on this GPU (TFLOP/s), the denominator for FP64 kernels
    (the pool's measured-peaks file lists HBM and bf16 only)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize(dev)
    best = 1e30
    for _ in range(5):
        s, t = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        t.record()
        t.synchronize()
        best = min(best, s.elapsed_time(t))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def ncu_traffic(kernel):
    """DRAM bytes per launch from the committed ncu summary, if one exists."""
    path = os.path.join(HERE, "profiles", f"{kernel}.txt")
    try:
        for line in open(path, encoding="utf-8"):
            if line.startswith("dram_bytes_per_launch_full_size:"):
                return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


# ---- CPU baseline: the oracle (C restatement of the reference's TS path) -------------

def cpu_step_estimate(v, e, blocks, step_stats, budget_s):
    """Times bounded samples of the oracle's step at full size and scales each
    phase by its exact operation count: gradient, energy and Gram assembly over a
    subset of edge rows (x E/rows), the (3V+k) Bunch-Kaufman LDL^T factor at a
    smaller order n_s (x (n/n_s)^3) and its solve (x (n/n_s)^2). Returns
    (seconds per step, description)."""
    sys.path.insert(0, os.path.join(HERE, "tests"))
    import oracle_lib as O
    from repulsive_test2_b200 import abi

    L = O.lib()
    V, E = len(v), len(e)
    vv = np.ascontiguousarray(v)
    ee = np.ascontiguousarray(e, dtype=np.int32)
    vp, ep = vv.ctypes.data_as(abi.dp), ee.ctypes.data_as(abi.ip)
    per = budget_s / 4.0

    def rows_time(fn):
        r = 8
        while True:
            t0 = time.perf_counter()
            fn(r)
            dt = time.perf_counter() - t0
            if dt > per / 4 or r >= E:
                return dt * E / r, r
            r = min(E, r * 4)

    g = np.zeros((V, 3))
    t_grad, r_g = rows_time(lambda r: L.tpeo_gradient_rows(vp, V, ep, E, 3.0, 6.0, 1e-10, 0, r,
                                                           g.ctypes.data_as(abi.dp)))
    t_en, r_e = rows_time(lambda r: L.tpeo_energy_rows(vp, V, ep, E, 3.0, 6.0, 1e-10, 0, r))
    A = np.zeros((V, V))
    t_asm, r_a = rows_time(lambda r: L.tpeo_assemble_a_rows(vp, V, ep, E, 3.0, 6.0, 1e-10, 0, r,
                                                            A.ctypes.data_as(abi.dp)))
    del A
    k = O.lib().tpeo_constraint_rows(abi.make_set(blocks)[0], len(blocks), E)
    n = 3 * V + k
    ns = 256
    rng = np.random.default_rng(0)
    while True:
        M = rng.standard_normal((ns, ns))
        M = M + M.T
        piv = np.zeros(ns, dtype=np.int32)
        t0 = time.perf_counter()
        L.tpeo_ldlt_factor(M.ctypes.data_as(abi.dp), ns, piv.ctypes.data_as(abi.ip))
        tf = time.perf_counter() - t0
        x = np.zeros(ns)
        rhs = rng.standard_normal(ns)
        t0 = time.perf_counter()
        L.tpeo_ldlt_solve(M.ctypes.data_as(abi.dp), ns, piv.ctypes.data_as(abi.ip),
                          rhs.ctypes.data_as(abi.dp), x.ctypes.data_as(abi.dp))
        ts = time.perf_counter() - t0
        if tf > per or ns >= min(4096, n):
            break
        ns = int(ns * 1.6)
    t_fac = tf * (n / ns) ** 3
    t_sol = ts * (n / ns) ** 2
    trials = max(1, int(step_stats.get("trials", 1)))
    iters = max(0, int(step_stats.get("projection_iterations", 1) or 0))
    # E0 + one energy per trial; one LDL^T solve for g~ plus one per projection
    # iterate of every trial (frozen); the structured residual is an O(n^2) matvec.
    total = t_grad + t_en * (1 + trials) + t_asm + t_fac + t_sol * (1 + trials * iters) + t_sol
    desc = (f"oracle (C restatement of the reference TS path, 1 thread), V={V}: gradient {r_g} of {E} "
            f"edge rows x{E / r_g:.0f}, energy {r_e} rows x{E / r_e:.0f} x(1+{trials} trials), "
            f"assembly {r_a} rows x{E / r_a:.0f}, Bunch-Kaufman LDL^T of order {ns} scaled to n={n} "
            f"by (n/ns)^3, its solve by (n/ns)^2")
    return total, desc, {"grad_s": t_grad, "energy_s": t_en, "assemble_s": t_asm, "factor_s": t_fac,
                         "solve_s": t_sol}


# ---- our arm ---------------------------------------------------------------------------

def run_repulsive(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    from repulsive_test2_b200 import abi
    from repulsive_test2_b200 import api as T

    v, e, blocks = workload(args.V)
    ctx = T.Context(local)
    ctx.topology(v, e)
    lib = ctx.lib
    arr, keep = abi.make_set(blocks)
    o = T._opts({"projectionMode": "frozen", "precision": args.precision})
    st = abi.tpe_step_stats()
    d_in = torch.from_numpy(v.copy()).to(dev)
    d_out = torch.empty_like(d_in)
    stream = torch.cuda.ExternalStream(lib.tpe_stream(ctx.ptr), device=dev)

    def dev_step():
        rc = lib.tpe_sobolev_step_device(ctx.ptr, d_in.data_ptr(), arr, len(blocks), C.byref(o),
                                         d_out.data_ptr(), C.byref(st), None)
        ctx.check(rc, "tpe_sobolev_step_device")

    for _ in range(args.warmup):
        dev_step()
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    lib.tpe_profile(ctx.ptr, 1)
    with ClockSampler(local) as clk:
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        t0.record(stream)
        for _ in range(args.steps):
            dev_step()
        t1.record(stream)
        torch.cuda.synchronize(dev)
    ms = t0.elapsed_time(t1)
    kms = (C.c_double * len(abi.KGROUPS))()
    kl = (C.c_int64 * (len(abi.KGROUPS) + 1))()
    lib.tpe_profile_read(ctx.ptr, kms, kl)
    lib.tpe_profile(ctx.ptr, 0)
    step_info = {"trials": st.trials_evaluated, "projection_iterations": st.projection_iterations,
                 "tau": st.tau, "accepted": st.accepted, "energy_before": st.energy_before,
                 "energy_after": st.energy}
    if dist:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    # e2e: the public host-buffer API (pinned host in/out, copies inside the region)
    pin_in = torch.from_numpy(v.copy()).pin_memory()
    pin_out = torch.empty_like(pin_in).pin_memory()
    vin = pin_in.numpy()
    vout = pin_out.numpy()
    inp = vin.ctypes.data_as(abi.dp)
    outp = vout.ctypes.data_as(abi.dp)

    def host_step():
        rc = lib.tpe_sobolev_step(ctx.ptr, inp, arr, len(blocks), C.byref(o), outp, C.byref(st), None, None)
        ctx.check(rc, "tpe_sobolev_step")

    host_step()
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        host_step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())

    if rank != 0:
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    V = args.V
    groups = abi.KGROUPS
    ms_g = {g: kms[i] for i, g in enumerate(groups)}
    nl = {g: kl[i] for i, g in enumerate(groups)}
    dom = max(ms_g, key=lambda g: ms_g[g])
    peaks = measured_peaks()
    fp64_peak = fp64_gemm_peak(torch, dev)
    steps = args.steps
    # algorithmic work per launch of the dominant group
    if dom == "cholesky":
        per_launch_flop = V ** 3 / 3.0  # one Cholesky of A_rho per step
        n_launch = steps
        roof = {"bound": "tensor", "unit": "TFLOP/s", "peak": fp64_peak,
                "peak_source": "cuBLAS FP64 GEMM measured in this run (no FP64 entry in MEASURED_PEAKS.json)",
                "kernel": "cholesky (potrf_diag+trsm_panel+syrk_update), per factorization",
                "work_per_launch": f"V^3/3 = {per_launch_flop:.3e} flop"}
        achieved = per_launch_flop * n_launch / (ms_g[dom] * 1e-3) / 1e12
    elif dom in ("gradient", "energy", "pair_weights"):
        P = len(e) * (len(e) - 3)
        fl = {"gradient": 2 * 4 * 110, "energy": 4 * 34, "pair_weights": 4 * 45}[dom]
        per_launch_flop = P * fl
        n_launch = max(1, nl[dom] // {"gradient": 2, "energy": 2, "pair_weights": 1}[dom])
        roof = {"bound": "tensor", "unit": "TFLOP/s", "peak": fp64_peak,
                "peak_source": "cuBLAS FP64 GEMM measured in this run (FP64 pipe reference)",
                "kernel": dom, "work_per_launch": f"{fl} flop x {P} ordered pairs"}
        achieved = per_launch_flop * n_launch / (ms_g[dom] * 1e-3) / 1e12
    else:
        per_launch_bytes = 8.0 * V * V * 2
        n_launch = max(1, nl[dom])
        roof = {"bound": "hbm", "unit": "GB/s", "peak": peaks.get("hbm_gbs", 6650.0),
                "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650",
                "kernel": dom, "work_per_launch": "16 V^2 bytes"}
        achieved = per_launch_bytes * n_launch / (ms_g[dom] * 1e-3) / 1e9
    roof["achieved"] = achieved
    roof["frac"] = achieved / roof["peak"] if roof["peak"] else None
    roof["traffic"] = ncu_traffic(dom)
    roof["avg_launch_ms"] = ms_g[dom] / max(1, n_launch)
    roof["group_ms"] = {g: round(ms_g[g], 3) for g in groups}
    roof["group_launches"] = {g: int(nl[g]) for g in groups}

    value = world * steps / (ms * 1e-3)
    e2e_value = world * steps / (e2e_ms * 1e-3)
    out = {
        "metric": METRIC,
        "value": value,
        "unit": "steps/s",
        "n_gpus": world,
        "steps": steps,
        "warmup": args.warmup,
        "ms_per_step": ms / steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32-mixed",
        "data": "synthetic: seeded random-walk knot (splitmix64/Box-Muller), no dataset",
        "config": {"workload": f"random-walk closed knot V=E={V}, [barycenter,totalLength], frozen projection, "
                               "analytical dE, one sobolevStepSet per step from the same input",
                   "V": V, "precision": args.precision, "parallelism": "replicas" if world > 1 else "single",
                   "l2": "working set larger than L2 (A and L are 537 MB each, pair matrix 1.07 GB)"},
        "step": step_info,
        "roofline": roof,
        "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": 8 * 3 * V,
                "d2h_bytes_per_step": 8 * 3 * V},
        "gpu_launches": int(kl[len(groups)]),
        "clocks": clk.summary(),
    }
    if not args.no_cpu_baseline and world == 1:
        t_cpu, desc, parts = cpu_step_estimate(v, e, blocks, step_info, args.cpu_budget)
        out["cpu_baseline"] = {"value": 1.0 / t_cpu, "unit": "steps/s", "cores": 1, "kind": "port",
                               "sample": desc, "phases_s": {k: round(x, 3) for k, x in parts.items()}}
    print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    v, e, blocks = workload(args.V)
    per_step = max(2.0, min(30.0, 150.0 / max(1, args.steps)))
    # warm-up: one small sample (the CPU has no compile/caching stage to warm)
    cpu_step_estimate(v, e, blocks, {"trials": 1, "projection_iterations": 1}, 1.0)
    t_total = 0.0
    desc = ""
    for _ in range(args.steps):
        t, desc, _parts = cpu_step_estimate(v, e, blocks, {"trials": 1, "projection_iterations": 1}, per_step)
        t_total += t
    value = args.steps / t_total
    out = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * t_total / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic: seeded random-walk knot (splitmix64/Box-Muller), no dataset",
        "config": {"workload": f"random-walk closed knot V=E={args.V}, [barycenter,totalLength], frozen projection, "
                               "analytical dE, one sobolevStepSet per step", "V": args.V},
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": 1, "kind": "port", "sample": desc},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_repulsive(args)


if __name__ == "__main__":
    main()
