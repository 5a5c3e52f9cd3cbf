#!/usr/bin/env python
"""Descent-step throughput of the constrained fractional-Sobolev step on B200.

Workload (the reference's precision-form configuration): a seeded random-walk
closed knot with V = E = 8192 (3-D Gaussian steps of sigma 1/sqrt(V), closed by
drift removal, total length 10), tangent-point alpha=3, beta=6, eps=1e-10,
constraint set [barycenter, totalLength] frozen at the initial curve, frozen
projection (the app's default), analytical dE. One step = one sobolevStepSet
(gradient, Gram assembly, structured saddle solve, Armijo line search with
back-projection); the timed loop is a descent trajectory, each step starting at
the previous step's output.

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


# Algorithmic flops per unordered disjoint edge pair (both orders), counted from
# the kernels' arithmetic with +, -, *, /, sqrt and rsqrt as one flop each and
# integer powers as their multiplies: the energy (4 endpoint pairs x 60 + 9),
# the adjoint gradient with its energy (4 x 163 + 141) and the Gram pair
# weights with their stencil (4 x 63 + 26).
FLOP_PER_UNORDERED_PAIR = {"energy": 249, "gradient": 793, "pair_weights": 278}


def max_over_ranks(ms, dist, device):
    """The slowest rank's time, on every rank (ms itself without a process group)."""
    if dist is None:
        return ms
    import torch

    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(steps, world, ms):
    """Whole-job throughput of `world` replicas: every rank's steps over the max time."""
    return world * steps / (ms * 1e-3)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="repulsive", choices=["repulsive", "reference"])
    p.add_argument("--V", type=int, default=8192)
    p.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of oracle work")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the per-edge, multi-curve batch and network measurements")
    p.add_argument("--network-steps", type=int, default=50)
    return p.parse_args()


def extras(args):
    """The other workload forms, each timed through the public API (host buffers,
    wall clock around synchronous calls): per-edge length constraints at V=8192
    (k = E + 3), a 64-curve batch of uneven sizes, and the 12 x 1024 loop
    network with pins and penalties."""
    from repulsive_test2_b200 import api as T
    from repulsive_test2_b200 import fixtures as F

    out = {}
    # per-edge length constraints at V=8192
    v, e = F.random_walk_knot(args.V, seed=1)
    ell = T.edgeLengths(v, e)
    blocks = [T.barycenterBlock(T.barycenterTarget(v, e)), T.edgeLengthsBlock(ell)]
    o = {"projectionMode": "frozen", "precision": "mixed", "trials": 8,
         "energyBefore": T.calculateEnergy(v, e)}
    o64 = dict(o, precision="fp64", trials=1)

    def one_step(opts):
        T.sobolevStepSet(v, e, None, blocks, opts)
        best, res = None, None
        for _ in range(2):
            t0 = time.perf_counter()
            res = T.sobolevStepSet(v, e, None, blocks, opts)
            dt_ = time.perf_counter() - t0
            best = dt_ if best is None else min(best, dt_)
        return best, res

    dt, r = one_step(o)
    dt64, r64 = one_step(o64)
    dt64b, _ = one_step(dict(o, precision="fp64"))  # FP64 with the same batched step sizes
    out["per_edge"] = {
        "workload": f"random-walk knot V=E={args.V}, [barycenter, edgeLengths] (k = {len(ell) + 3}), one step",
        "ms_per_step": dt * 1e3, "fp64_ms_per_step": dt64 * 1e3, "speedup_vs_fp64": dt64 / dt,
        "fp64_batched_ms_per_step": dt64b * 1e3,
        "tau": r["stats"]["tau"], "fp64_tau": r64["stats"]["tau"],
        "saddle_residual": r["stats"]["residual"],
        "energy_rel_err_vs_fp64": abs(r["energy"] - r64["energy"]) / abs(r64["energy"]),
        "vertices_rel_err_vs_fp64": float(np.linalg.norm(r["vertices"] - r64["vertices"]) /
                                          np.linalg.norm(r64["vertices"])),
        "path": "explicit inverses of A_rho and of the k x k Schur complement (k > 64): mixed = "
                "recursive Cholesky and triangular inverse with FP64-class products on the int8 tensor "
                "cores (eight 8-bit digits per element, exact int32 digit GEMMs); fp64 = the same on the "
                "FP64 tensor cores (DMMA)"}
    # 64-curve batch
    curves = F.batch_curves(count=64, vmin=256, vmax=4096, seed=3)
    sets = [[T.barycenterBlock(T.barycenterTarget(cv, ce)), T.totalLengthBlock(T.totalLength(cv, ce))]
            for cv, ce in curves]
    ob = {"projectionMode": "frozen", "precision": "mixed", "trials": 8}
    b = T.Batch(curves)
    xs = [cv for cv, _ in curves]
    b.step(xs, sets, ob)
    t0 = time.perf_counter()
    nb = 3
    for _ in range(nb):
        b.step(xs, sets, ob)
    dtb = (time.perf_counter() - t0) / nb
    t0 = time.perf_counter()
    per_curve = []
    for (cv, ce), st_ in zip(curves, sets):
        t1 = time.perf_counter()
        T.sobolevStepSet(cv, ce, None, st_, ob)
        per_curve.append((len(cv), time.perf_counter() - t1))
    dts = time.perf_counter() - t0
    # the sequential steps' time by size octave: where the batch's time goes
    octaves = {}
    for nv_, dtc in per_curve:
        lo_ = 256
        while lo_ * 2 <= nv_ and lo_ < 2048:
            lo_ *= 2
        key = f"V{lo_}-{2 * lo_}"
        octaves.setdefault(key, [0, 0.0])
        octaves[key][0] += 1
        octaves[key][1] += dtc * 1e3
    b.close()
    out["batch"] = {"workload": "64 curves, V log-uniform in [256, 4096] (trefoil / torus knots / random "
                                "walks), [barycenter, totalLength], mixed, 8 step sizes per projection batch",
                    "curve_steps_per_s": 64 / dtb, "ms_per_batch_step": dtb * 1e3,
                    "sequential_curve_steps_per_s": 64 / dts,
                    "sequential_ms_by_octave": {k: {"curves": c, "ms": round(t_, 2)}
                                                for k, (c, t_) in sorted(octaves.items())}}
    # loop network
    PEN = {"totalLength": 1.0, "lengthDiff": 10.0, "field": {"weight": 5.0, "X": [0.5, 1.0, 0.0]}}
    nv, ne = F.loop_network(loops=12, n=1024, junctions=8, seed=5)
    pins = F.seeded_pins(len(nv), 16, seed=11)
    nbk = [T.barycenterBlock(T.barycenterTarget(nv, ne)), T.edgeLengthsBlock(T.edgeLengths(nv, ne))]
    nbk += [T.pointBlock(int(p_), nv[p_]) for p_ in pins]
    net = {"workload": f"12 x 1024 random-walk loops, 8 Y-junctions (V={len(nv)}, E={len(ne)}), 16 pins, "
                       "penalties (1, 10, 5, X=(0.5,1,0)), [barycenter, edgeLengths, 16 points]",
           "steps": args.network_steps}
    finals = {}
    for prec in ("fp64", "mixed"):
        x = nv.copy()
        acc = 0
        t0 = time.perf_counter()
        for _ in range(args.network_steps):
            rr = T.sobolevStepSet(x, ne, None, nbk, {"projectionMode": "frozen", "precision": prec,
                                                    "penalties": PEN})
            if rr["accepted"]:
                x = rr["vertices"]
                acc += 1
        dtn = time.perf_counter() - t0
        finals[prec] = x
        net[prec] = {"ms_per_step": dtn * 1e3 / max(1, args.network_steps), "accepted": acc,
                     "energy_last": rr["energy"]}
    net["mixed_vs_fp64_vertices_rel_err"] = float(np.linalg.norm(finals["mixed"] - finals["fp64"]) /
                                                  np.linalg.norm(finals["fp64"]))
    net["speedup_vs_fp64"] = net["fp64"]["ms_per_step"] / net["mixed"]["ms_per_step"]
    out["network"] = net
    # sizes that are not a multiple of 128 (the mixed factor pads to the next multiple)
    rag = {"workload": "random-walk knot, [barycenter, totalLength], mixed, 8 step sizes per batch; one "
                       "step from the initial curve, best of 3 after one warm-up (wall time, host API)"}
    for Vr in (4096, 4097, 6000):
        rv, re_ = F.random_walk_knot(Vr, seed=1)
        rb = [T.barycenterBlock(T.barycenterTarget(rv, re_)), T.totalLengthBlock(T.totalLength(rv, re_))]
        ro = {"projectionMode": "frozen", "precision": "mixed", "trials": 8,
              "energyBefore": T.calculateEnergy(rv, re_)}
        T.sobolevStepSet(rv, re_, None, rb, ro)
        best = None
        for _ in range(3):
            t0 = time.perf_counter()
            T.sobolevStepSet(rv, re_, None, rb, ro)
            dt_ = time.perf_counter() - t0
            best = dt_ if best is None else min(best, dt_)
        rag[f"V{Vr}_ms"] = best * 1e3
    rag["ratio_4097_over_4096"] = rag["V4097_ms"] / rag["V4096_ms"]
    out["ragged_sizes"] = rag
    # Barnes-Hut energy (the hierarchical path) against the exact GPU energy on a
    # smooth curve far larger than the step's V
    bh = {"workload": "closed trefoil (the stage-2 oracle's check curve), theta 0.5, theta_t 0.75, leaf 8; "
                      "wall time of the public calls (tree and block lists built on the host, traversal and "
                      "products on the device); bct_high: the high-order kernel product against theta = 0"}
    for n in (32768, 131072):
        tt = np.linspace(0.0, 2.0 * np.pi, n, endpoint=False)
        tv = np.stack([np.sin(tt) + 2.0 * np.sin(2.0 * tt), np.cos(tt) - 2.0 * np.cos(2.0 * tt),
                       -np.sin(3.0 * tt)], axis=1) * 0.25
        te = np.stack([np.arange(n), (np.arange(n) + 1) % n], axis=1).astype(np.int32)
        T.calculateEnergy(tv, te)
        t0 = time.perf_counter()
        ex = T.calculateEnergy(tv, te)
        t_ex = time.perf_counter() - t0
        T.bhEnergy(tv, te, theta=0.5, leafSize=8, thetaT=0.75)
        t0 = time.perf_counter()
        eb, stb = T.bhEnergy(tv, te, theta=0.5, leafSize=8, thetaT=0.75)
        t_bh = time.perf_counter() - t0
        bh[f"E{n}"] = {"exact_ms": t_ex * 1e3, "bh_ms": t_bh * 1e3, "rel_err": abs(eb - ex) / abs(ex),
                       "direct_pairs_fraction": stb["direct_pairs"] / float(n) ** 2, **stb}
        if n == 32768:
            # the block-cluster-tree product of the high-order kernel against theta = 0 (exact)
            psi = np.sin(np.arange(n) * 0.61) + 0.2
            t0 = time.perf_counter()
            k_ex, _ = T.bctMatvec(tv, te, psi, "high", theta=0.0, leafSize=8)
            t_kex = time.perf_counter() - t0
            T.bctMatvec(tv, te, psi, "high", theta=0.5, leafSize=8, thetaT=0.75)
            t0 = time.perf_counter()
            k_bct, stk = T.bctMatvec(tv, te, psi, "high", theta=0.5, leafSize=8, thetaT=0.75)
            t_k = time.perf_counter() - t0
            bh[f"E{n}"]["bct_high"] = {"exact_ms": t_kex * 1e3, "bct_ms": t_k * 1e3,
                                       "rel_err": float(np.linalg.norm(k_bct - k_ex) / np.linalg.norm(k_ex)),
                                       **stk}
    out["bh"] = bh
    return out


def bench_config(V):
    """The workload both arms run (same dict in the reference arm's line)."""
    return {"workload": f"random-walk closed knot V=E={V}, [barycenter,totalLength] frozen at the initial "
                        "curve, frozen projection, analytical dE; a descent trajectory, each step starting "
                        "at the previous output with its energy as energyBefore (the app's loop)",
            "V": V,
            "l2": "working set larger than L2 (A is 537 MB, the FP32 factor and its inverse 1.6 GB)"}


def host_info():
    model = ""
    try:
        for line in open("/proc/cpuinfo", encoding="utf-8"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"cpu": model, "logical_cores": os.cpu_count()}


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

# Line-search work of one step on this workload, as the GPU FP64 step does it
# from the initial curve: 7 step sizes tried (tau = 1 .. 2^-6), the first 5
# projections fail at the 8-correction cap, the last 2 converge in 3 and are
# the 2 energy evaluations (E0 comes in as energyBefore).
LS_ENERGIES = 2
LS_SOLVES = 5 * 8 + 2 * 3


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
    energies = int(step_stats.get("energies", LS_ENERGIES))
    solves = int(step_stats.get("solves", LS_SOLVES))
    # the line search's energies, one LDL^T solve for g~ plus one per projection
    # correction (frozen), and the structured residual (an O(n^2) matvec ~ a solve)
    total = t_grad + t_en * energies + t_asm + t_fac + t_sol * (1 + solves) + t_sol
    desc = (f"oracle (C restatement of the reference TS path, 1 thread), V={V}: gradient {r_g} of {E} "
            f"edge rows x{E / r_g:.0f}, energy {r_e} rows x{E / r_e:.0f} x{energies} line-search "
            f"evaluations, assembly {r_a} rows x{E / r_a:.0f}, Bunch-Kaufman LDL^T of order {ns} scaled "
            f"to n={n} by (n/ns)^3, its solve by (n/ns)^2 x{1 + solves}")
    return total, desc, {"grad_s": t_grad, "energy_s": t_en, "assemble_s": t_asm, "factor_s": t_fac,
                         "solve_s": t_sol}


# ---- our arm ---------------------------------------------------------------------------

def step_opts(T, precision):
    """mixed+batched: FP32 tensor-core factor + FP64 CG, 8 step sizes projected per
    batch; plain FP64: FP64 factorization, one step size at a time."""
    return T._opts({"projectionMode": "frozen", "precision": precision,
                    "trials": 8 if precision == "mixed" else 1})


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
    st = abi.tpe_step_stats()
    stream = torch.cuda.ExternalStream(lib.tpe_stream(ctx.ptr), device=dev)
    params = abi.tpe_params(3.0, 6.0, 1e-10)
    e_init = C.c_double(0.0)
    ctx.check(lib.tpe_energy(ctx.ptr, np.ascontiguousarray(v).ctypes.data_as(abi.dp), C.byref(params),
                             C.byref(e_init)), "tpe_energy")
    E0 = e_init.value
    d_init = torch.from_numpy(v.copy()).to(dev)
    bufs = [torch.empty_like(d_init), torch.empty_like(d_init)]

    def dev_trajectory(o, nsteps, log=None):
        """nsteps descent steps from the initial curve; step i starts at the
        output of step i-1 with its energy as energyBefore (the app's loop)."""
        bufs[0].copy_(d_init)
        cur, nxt = 0, 1
        e_before = E0
        for _ in range(nsteps):
            o.has_energy_before = 1
            o.energy_before = e_before
            rc = lib.tpe_sobolev_step_device(ctx.ptr, bufs[cur].data_ptr(), arr, len(blocks), C.byref(o),
                                             bufs[nxt].data_ptr(), C.byref(st), None)
            ctx.check(rc, "tpe_sobolev_step_device")
            if log is not None:
                log.append({"tau": st.tau, "trials": st.trials_evaluated, "accepted": st.accepted,
                            "refine": st.refine_iterations, "energy": st.energy})
            if st.accepted:
                cur, nxt = nxt, cur
                e_before = st.energy

    def timed(o, nsteps, log=None, profile=False):
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()
        if profile:
            lib.tpe_profile(ctx.ptr, 1)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        t0.record(stream)
        dev_trajectory(o, nsteps, log)
        t1.record(stream)
        torch.cuda.synchronize(dev)
        return max_over_ranks(t0.elapsed_time(t1), dist, dev)

    o_mix = step_opts(T, args.precision)
    o_64 = step_opts(T, "fp64")
    for _ in range(args.warmup):
        dev_trajectory(o_mix, 1)
        dev_trajectory(o_64, 1)
    log_mix, log_64 = [], []
    with ClockSampler(local) as clk:
        lib.tpe_profile(ctx.ptr, 0)  # zeroes the launch counter; no per-group events
        ms = timed(o_mix, args.steps, log_mix)
        kl_timed = (C.c_int64 * (len(abi.KGROUPS) + 1))()
        lib.tpe_profile_read(ctx.ptr, None, kl_timed)
        ms64 = timed(o_64, args.steps, log_64)
    # Per-group device time for the roofline: the same trajectory once more with
    # CUDA events around each kernel group (kept out of the headline timing).
    ms_prof = timed(o_mix, args.steps, None, profile=True)
    kms = (C.c_double * len(abi.KGROUPS))()
    kl = (C.c_int64 * (len(abi.KGROUPS) + 1))()
    lib.tpe_profile_read(ctx.ptr, kms, kl)
    lib.tpe_profile(ctx.ptr, 0)

    # e2e: the public host-buffer API (pinned host in/out, copies inside the region)
    pin = [torch.from_numpy(v.copy()).pin_memory(), torch.empty_like(torch.from_numpy(v)).pin_memory()]
    hp = [pin[0].numpy().ctypes.data_as(abi.dp), pin[1].numpy().ctypes.data_as(abi.dp)]

    def host_trajectory(o, nsteps):
        pin[0].copy_(torch.from_numpy(v))
        cur, nxt = 0, 1
        e_before = E0
        for _ in range(nsteps):
            o.has_energy_before = 1
            o.energy_before = e_before
            rc = lib.tpe_sobolev_step(ctx.ptr, hp[cur], arr, len(blocks), C.byref(o), hp[nxt], C.byref(st),
                                      None, None)
            ctx.check(rc, "tpe_sobolev_step")
            if st.accepted:
                cur, nxt = nxt, cur
                e_before = st.energy

    host_trajectory(o_mix, 1)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    host_trajectory(o_mix, args.steps)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), dist, dev)

    # Mixed against FP64 along the trajectory. (a) Fed the same iterate: at every
    # iterate x_i of the FP64 trajectory both steps start from x_i with E(x_i) as
    # energyBefore, so each step's error is its own. (b) Free-running: the two
    # timed trajectories side by side (their iterates drift apart once an
    # accepted step size differs).
    acc = {}
    if rank == 0:
        x, eb = v.copy(), E0
        per = []
        for i in range(args.steps):
            base = {"projectionMode": "frozen", "energyBefore": eb, "collectField": True}
            rf = T.sobolevStepSet(x, e, None, blocks, dict(base, precision="fp64", trials=1))
            rm = T.sobolevStepSet(x, e, None, blocks, dict(base, precision=args.precision,
                                                             trials=int(o_mix.trials)))
            gm, gf = rm["descentField"], rf["descentField"]
            per.append({"energy": abs(rm["energy"] - rf["energy"]) / abs(rf["energy"]),
                        "g": float(np.linalg.norm(gm - gf) / np.linalg.norm(gf)),
                        "x": float(np.linalg.norm(rm["vertices"] - rf["vertices"]) / np.linalg.norm(rf["vertices"])),
                        "tau_equal": rm["stats"]["tau"] == rf["stats"]["tau"],
                        "cg": rm["stats"]["refineIterations"], "residual": rm["stats"]["residual"]})
            if rf["accepted"]:
                x, eb = rf["vertices"], rf["energy"]
        acc = {"steps": len(per),
               "energy_rel_err_max": max(p_["energy"] for p_ in per),
               "projected_gradient_rel_err_max": max(p_["g"] for p_ in per),
               "vertices_rel_err_max": max(p_["x"] for p_ in per),
               "tau_equal_steps": sum(p_["tau_equal"] for p_ in per),
               "saddle_residual_max": max(p_["residual"] for p_ in per),
               "cg_iterations": [p_["cg"] for p_ in per],
               "method": "both solves from every iterate of the FP64 trajectory (same x_i, same "
                         "energyBefore); errors of the mixed step against the FP64 step"}

    if rank != 0:
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    V = args.V
    groups = abi.KGROUPS
    ms_g = {g: kms[i] for i, g in enumerate(groups)}
    nl = {g: kl[i] for i, g in enumerate(groups)}
    # The gradient runs beside the factorization on two fifths of the SMs (its group
    # time is the stream3 span, not a full-GPU kernel time): the roofline is taken
    # for the dominant group on the main stream, the gradient reported apart.
    dom = max((g for g in ms_g if g != "gradient" or args.precision != "mixed"), key=lambda g: ms_g[g])
    peaks = measured_peaks()
    fp64_peak = fp64_gemm_peak(torch, dev)
    steps = args.steps
    P = len(e) * (len(e) - 3)
    if dom in ("gradient", "energy", "pair_weights"):
        fl = FLOP_PER_UNORDERED_PAIR[dom]
        per_launch_flop = P / 2 * fl
        n_launch = max(1, nl[dom] // {"gradient": 2, "energy": 2, "pair_weights": 1}[dom])
        roof = {"bound": "tensor", "unit": "TFLOP/s", "peak": fp64_peak,
                "peak_source": "cuBLAS FP64 GEMM measured in this run (the FP64 pipe; MEASURED_PEAKS.json "
                               "lists HBM and bf16 only)",
                "kernel": dom, "work_per_launch": f"{fl} flop x {P // 2} unordered pairs"}
        achieved = per_launch_flop * n_launch / (ms_g[dom] * 1e-3) / 1e12
    elif dom == "cholesky":
        per_launch_flop = V ** 3 / 3.0
        n_launch = steps
        tf32 = peaks.get("bf16_tflops", 1590.0) / 2.0
        if args.precision == "mixed":
            roof = {"bound": "tensor", "unit": "TFLOP/s", "peak": tf32 / 3.0,
                    "peak_source": "MEASURED_PEAKS.json bf16_tflops / 2 (TF32) / 3 (3xTF32 products per "
                                   "algorithmic FMA)",
                    "kernel": "FP32 Cholesky of the scaled A_rho (potrf128 + tcgen05 3xTF32 GEMMs), per "
                              "factorization", "work_per_launch": f"V^3/3 = {per_launch_flop:.3e} flop"}
        else:
            roof = {"bound": "tensor", "unit": "TFLOP/s", "peak": fp64_peak,
                    "peak_source": "cuBLAS FP64 GEMM measured in this run",
                    "kernel": "FP64 Cholesky (DMMA)", "work_per_launch": f"V^3/3 = {per_launch_flop:.3e} flop"}
        achieved = per_launch_flop * n_launch / (ms_g[dom] * 1e-3) / 1e12
    else:
        per_launch_bytes = 8.0 * V * V
        n_launch = max(1, nl[dom])
        roof = {"bound": "hbm", "unit": "GB/s", "peak": peaks.get("hbm_gbs", 6650.0),
                "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650",
                "kernel": dom, "work_per_launch": "8 V^2 bytes"}
        achieved = per_launch_bytes * n_launch / (ms_g[dom] * 1e-3) / 1e9
    roof["achieved"] = achieved
    roof["frac"] = achieved / roof["peak"] if roof["peak"] else None
    roof["traffic"] = ncu_traffic(dom)
    roof["avg_launch_ms"] = ms_g[dom] / max(1, n_launch)
    roof["group_ms"] = {g: round(ms_g[g], 3) for g in groups}
    if args.precision == "mixed" and nl["gradient"] > 0:
        nsm = torch.cuda.get_device_properties(dev).multi_processor_count
        gsm = int(os.environ.get("TPE_GRAD_SMS", nsm * 2 // 5))
        g_ach = P / 2 * FLOP_PER_UNORDERED_PAIR["gradient"] * max(1, nl["gradient"] // 2) / (ms_g["gradient"] * 1e-3) / 1e12
        roof["concurrent_gradient"] = {
            "sms": gsm, "achieved": g_ach, "peak_on_its_sms": fp64_peak * gsm / nsm,
            "frac": g_ach / (fp64_peak * gsm / nsm) if fp64_peak else None, "unit": "TFLOP/s",
            "note": "adjoint gradient on stream3, bounded to `sms` SMs while the factorization runs; "
                    "the peak is the measured cuBLAS FP64 GEMM rate (DMMA), scaled to these SMs, "
                    "while the gradient runs on the FP64 FMA pipe"}
    roof["group_pass_ms_per_step"] = ms_prof / steps
    roof["group_pass"] = ("a second pass over the same trajectory with CUDA events around each kernel "
                          "group on the launching streams; the headline ms_per_step is the pass "
                          "without them")
    roof["group_launches"] = {g: int(nl[g]) for g in groups}

    value = replica_value(steps, world, ms)
    value64 = replica_value(steps, world, ms64)
    e2e_value = replica_value(steps, world, e2e_ms)

    def traj(log):
        return {"accepted": sum(x["accepted"] for x in log),
                "energy_evaluations": sum(x["trials"] for x in log),
                "taus": [x["tau"] for x in log], "cg_iterations": [x["refine"] for x in log],
                "energy_last": log[-1]["energy"] if log else None}

    # free-running: the two timed trajectories (b), beside the FP64 trajectory
    # from a start perturbed by 1e-12 relative (the descent map's own sensitivity)
    split = next((i for i, (a, b) in enumerate(zip(log_mix, log_64)) if a["tau"] != b["tau"]), None)
    traj_cmp = {"first_step_with_different_tau": split,
                "energy_last_rel_diff": (abs(log_mix[-1]["energy"] - log_64[-1]["energy"]) / abs(log_64[-1]["energy"])
                                         if log_mix and log_64 else None),
                "method": "the two timed trajectories, each step from its own previous output"}
    if rank == 0:
        rng = np.random.default_rng(0)
        xp = v + 1e-12 * np.linalg.norm(v) / np.sqrt(v.size) * rng.standard_normal(v.shape)
        ebp = T.calculateEnergy(xp, e)
        taus_p = []
        for _ in range(args.steps):
            r = T.sobolevStepSet(xp, e, None, blocks, {"projectionMode": "frozen", "energyBefore": ebp,
                                                       "precision": "fp64", "trials": 1})
            taus_p.append(r["stats"]["tau"])
            if r["accepted"]:
                xp, ebp = r["vertices"], r["energy"]
        traj_cmp["fp64_from_start_perturbed_1e-12"] = {
            "taus": taus_p,
            "first_step_with_different_tau": next((i for i, (a, b) in enumerate(zip(taus_p, log_64))
                                                   if a != b["tau"]), None),
            "note": "the FP64 step itself, from a start 1e-12 away: free-running trajectories separate "
                    "after a few steps whatever the solve (a relative difference grows 10-100x per step)"}

    # Key order: the long blocks first, the metric's comparison last (the end of
    # the line is what a truncated log shows).
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
        "dtype": "f64+tf32x3" if args.precision == "mixed" else "f64",
        "data": "synthetic: seeded random-walk knot (splitmix64/Box-Muller), no dataset",
        "config": bench_config(V),
        "arm": {"precision": args.precision,
                "line_search": "8 step sizes projected per batch" if args.precision == "mixed" else "sequential",
                "parallelism": "replicas" if world > 1 else "single"},
        "roofline": roof,
        "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": 8 * 3 * V,
                "d2h_bytes_per_step": 8 * 3 * V},
        "gpu_launches": int(kl_timed[len(groups)]),
        "clocks": clk.summary(),
    }
    if not args.no_extras and world == 1:
        out["extras"] = extras(args)
    if not args.no_cpu_baseline and world == 1:
        t_cpu, desc, parts = cpu_step_estimate(v, e, blocks, {}, args.cpu_budget)
        out["cpu_baseline"] = {"value": 1.0 / t_cpu, "unit": "steps/s", "cores": 1, "kind": "port",
                               "estimate": True, "sample": desc, "host": host_info(),
                               "phases_s": {k: round(x, 3) for k, x in parts.items()}}
    out["trajectory"] = traj(log_mix)
    out["fp64"] = {"value": value64, "unit": "steps/s", "ms_per_step": ms64 / steps,
                   "config": "plain FP64 GPU step: FP64 Cholesky, one step size at a time",
                   "trajectory": traj(log_64)}
    out["trajectory_vs_fp64"] = traj_cmp
    out["accuracy_vs_fp64"] = acc
    out["speedup_vs_fp64"] = value / value64
    print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def oracle_full_step(V):
    """Wall time of one whole oracle step (the reference's algorithm, 1 thread)
    on the same workload at a size it finishes in about a minute."""
    sys.path.insert(0, os.path.join(HERE, "tests"))
    import oracle_lib as O
    from repulsive_test2_b200 import abi

    v, e, blocks = workload(V)
    o = O.default_opts(projection_mode=abi.PROJECTION_FROZEN, has_energy_before=1,
                       energy_before=O.energy(v, e))
    t0 = time.perf_counter()
    rc, _out, st, _f = O.sobolev_step(v, e, blocks, o)
    dt = time.perf_counter() - t0
    return dt, {"rc": rc, "tau": st.tau, "trials_evaluated": st.trials_evaluated,
                "projection_iterations": st.projection_iterations}


def run_reference(args):
    """The reference's CPU path (its algorithm restated in C, single-threaded like
    the TypeScript it restates) on this workload. A whole V=8192 oracle step
    takes 17-23 minutes, so each of the K steps is a bounded sample of it:
    per-phase row samples of the pair work and a Bunch-Kaufman LDL^T at a smaller
    order, scaled by exact operation counts to one full step (an estimate, and
    labelled so). The model is checked in the same run against one whole oracle
    step timed at V=2048."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    t_start = time.perf_counter()
    v, e, blocks = workload(args.V)
    per_step = max(2.0, min(30.0, 150.0 / max(1, args.steps)))
    for _ in range(args.warmup):
        cpu_step_estimate(v, e, blocks, {}, 0.5)
    t_total = 0.0
    desc = ""
    ests = []
    for _ in range(args.steps):
        t, desc, _parts = cpu_step_estimate(v, e, blocks, {}, per_step)
        ests.append(t)
        t_total += t
    value = args.steps / t_total
    # the model against one whole step at V=2048
    check = {}
    if args.V > 2048:
        vs, es, bs = workload(2048)
        model_s, _d, _p = cpu_step_estimate(vs, es, bs, {}, per_step)
        full_s, info = oracle_full_step(2048)
        check = {"V": 2048, "measured_full_step_s": full_s, "model_s": model_s,
                 "model_over_measured": model_s / full_s, "oracle_step": info}
    wall = time.perf_counter() - t_start
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
        "config": bench_config(args.V),
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": 1, "kind": "port", "estimate": True,
                         "sample": desc + f"; {args.steps} such samples, one per step",
                         "host": host_info()},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "estimate": {"kind": "estimate",
                     "note": "each step's time is a full V=8192 step extrapolated from bounded samples, "
                             "so steps x ms_per_step exceeds the wall time of this run",
                     "wall_s": wall, "per_step_estimates_s": [round(x, 1) for x in ests],
                     "model_check": check},
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
