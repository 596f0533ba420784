"""Benchmark: PCG+GMG solves/s at 5.4M DOF (192x96x96 hex8 cantilever) to
a relative residual of 1e-8, mixed FP32/FP64 against plain FP64 on the same
GPU, with the matrix-free apply's achieved HBM bandwidth.

One step = one FE solve from U = 0 (the reference's KSPSolve,
FEAnalysis.cpp:673) plus the compliance and its filtered sensitivity
(Compliance.cpp:15-57), with the GMG hierarchy already set up for the
design -- the split the reference's own timer uses (FEAnalysis.cpp:707-710).
`e2e` is the whole design iteration through the C ABI with host buffers:
design upload, MatIntFnc, FEAssemble/PCSetUp, the solve, the sensitivity
and the download of C and dC/dx.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

For N > 1 (torchrun), every rank solves its own replica of the workload:
the path does not shard, so there is no data-path collective; the timing
is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = ("PCG+GMG solves/s at 5.4M DOF to 1e-8: mixed FP32/FP64 vs FP64 "
          "GPU; apply GB/s")
UNIT = "solves/s"
CONFIG = "cfg1"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-multi-rhs", action="store_true")
    ap.add_argument("--no-buckling", action="store_true")
    ap.add_argument("--no-oc", action="store_true")
    # profiling case: set up `--config` and launch one operation `--reps`
    # times with nothing else around it (for ncu captures; prints no line);
    # --config also selects the reference arm's problem (default 192x96x96)
    ap.add_argument("--kernel", default=None,
                    choices=["apply32", "apply64", "vcycle32", "vcycle64",
                             "solve_mixed", "solve_fp64", "mma", "setup", "setup_mixed",
                             "level1_32", "level1_32_stencil"])
    ap.add_argument("--config", default=CONFIG)
    ap.add_argument("--reps", type=int, default=3)
    # profiling cases: issue the CG iterations from the host instead of the
    # device-side loop graph, so that a profiler lists every kernel launch
    ap.add_argument("--no-graph", action="store_true")
    return ap.parse_args()


# ----------------------------------------------------------------- helpers

def dist_setup(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def measured_peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def committed_traffic(name):
    """dram bytes per launch from a committed ncu summary line
    `dram_bytes_per_launch: <int>` in profiles/<name>, else None."""
    p = os.path.join(HERE, "profiles", name)
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            if line.strip().startswith("dram_bytes_per_launch:"):
                try:
                    return int(float(line.split(":", 1)[1]))
                except ValueError:
                    return None
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.file = None

    def __enter__(self):
        self.skip = 0
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
            return self
        # the sampler takes a moment to start: wait (at most 5 s) for its
        # first row, and count only the rows written after this point, so
        # every sample used falls inside the timed region
        t_end = time.perf_counter() + 5.0
        while time.perf_counter() < t_end and self.proc.poll() is None:
            self.file.flush()
            with open(self.file.name) as f:
                n = sum(1 for r in f if r.strip())
            if n > 0:
                self.skip = n
                break
            time.sleep(0.01)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.proc or not self.file:
            return None
        self.file.flush()
        with open(self.file.name) as f:
            rows = [r.strip().split(", ") for r in f if r.strip()][self.skip:]
        os.unlink(self.file.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except ValueError:
                continue
            for k, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(k)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def build_problem(T, P, cfg):
    c = P.CONFIGS[cfg]
    t = T.TopOpt(c["nel"], rmin=c["rmin"], mg_levels=c["levels"])
    P.apply_bcs(t, P.bcs(cfg))
    t.FEInitialize()
    return t


# -------------------------------------------------------------- our arm

def run_ours(args, rank, world, local):
    import torch

    import topopt3d_b200 as T
    from topopt3d_b200 import problems as P

    dev = torch.device("cuda", local)
    # a non-default stream: handle 0 would select the library's own stream
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    cfg = P.CONFIGS[CONFIG]
    nel = cfg["nel"]
    ne, nn = int(np.prod(nel)), int(np.prod([n + 1 for n in nel]))
    x = P.design(CONFIG)

    t = build_problem(T, P, CONFIG)
    t.set_stream(stream.cuda_stream)
    x_dev = torch.tensor(x, device=dev)
    t.MatIntFnc(x_dev)
    mixed = T.default_opts(precision=T.PREC_MIXED)
    fp64 = T.default_opts(precision=T.PREC_FP64)
    t0 = time.perf_counter()
    t.FEAssemble(mixed)
    torch.cuda.synchronize(dev)
    setup_ms = (time.perf_counter() - t0) * 1e3
    # steady state: the hierarchy rebuilt for the same design (the per-
    # iteration cost of FEAssemble/PCSetUp in an optimisation loop), for
    # the mixed form and for the FP64 form (FP64 Chebyshev bounds)
    ev_a, ev_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def setup_time(opts):
        ts = []
        for _ in range(3):
            ev_a.record(stream)
            t.FEAssemble(opts)
            ev_b.record(stream)
            torch.cuda.synchronize(dev)
            ts.append(ev_a.elapsed_time(ev_b))
        return statistics.median(ts)

    setup_steady_fp64 = setup_time(fp64)
    setup_steady_ms = setup_time(mixed)   # leaves the mixed-form hierarchy

    zeros_u = torch.zeros(3 * nn, dtype=torch.float64, device=dev)
    dc = torch.zeros(ne, dtype=torch.float64, device=dev)
    infos = []

    def step(opts):
        t.set("U", zeros_u)
        info = t.FESolve(opts)
        C, _, _ = t.compliance(out=dc)
        infos.append((info, C))

    def timed(opts, k, w, sample_clocks=False):
        for _ in range(w):
            step(opts)
        barrier(world)
        torch.cuda.synchronize(dev)
        infos.clear()
        l0 = T.load().tpo_kernel_launches()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        sampler = ClockSampler(local) if sample_clocks else None
        if sampler:
            sampler.__enter__()
        ev0.record(stream)
        for _ in range(k):
            step(opts)
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        if sampler:
            sampler.__exit__(None, None, None)
        barrier(world)
        ms = ev0.elapsed_time(ev1)
        launches = T.load().tpo_kernel_launches() - l0
        return ms, launches, (sampler.summary() if sampler else None)

    ms_mx, launches, clocks = timed(mixed, args.steps, args.warmup, sample_clocks=True)
    info_mx = infos[-1]
    # the last timed step's solution, for the comparison with the oracle
    sol_mx = (t.U, info_mx[1], dc.cpu().numpy())
    t.FEAssemble(fp64)   # the FP64 form on its own (FP64) hierarchy
    ms_64, _, _ = timed(fp64, args.steps, args.warmup)
    info_64 = infos[-1]
    sol_64 = (t.U, info_64[1], dc.cpu().numpy())
    ms_mx = max_over_ranks(ms_mx, world)
    ms_64 = max_over_ranks(ms_64, world)
    value = world * args.steps / (ms_mx / 1e3)
    value_64 = world * args.steps / (ms_64 / 1e3)

    # roofline of the dominant kernel: the FP32 matrix-free apply, timed
    # launch by launch on the library's stream with an L2 flush between
    peak, peak_kind = measured_peaks()
    u64 = torch.randn(3 * nn, dtype=torch.float64, device=dev)
    y64 = torch.empty_like(u64)
    u32, y32 = u64.float(), torch.empty(3 * nn, dtype=torch.float32, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    lib = T.load()
    import ctypes as C
    durs = {}
    for name in ("fp32", "fp64"):
        ds = []
        for i in range(12):
            # a device-side wait first, so the launches below are queued
            # before the GPU reaches them and no host gap enters the timing
            torch.cuda._sleep(200000)
            flush.fill_(float(i))          # evict u, y, E from L2
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            if name == "fp64":
                t.apply(u64, y64, precision=T.PREC_FP64)
            else:
                rc = lib.tpo_apply_f32(t._h, C.c_void_p(u32.data_ptr()),
                                       C.c_void_p(y32.data_ptr()))
                assert rc == 0
            e1.record(stream)
            torch.cuda.synchronize(dev)
            ds.append(e0.elapsed_time(e1))
        durs[name] = statistics.median(ds[2:])
    bytes32 = 3 * nn * 4 * 2 + ne * 4 + nn          # u, y, E, fixed mask
    bytes64 = 3 * nn * 8 * 2 + ne * 8 + nn
    achieved32 = bytes32 / (durs["fp32"] * 1e-3) / 1e9
    achieved64 = bytes64 / (durs["fp64"] * 1e-3) / 1e9
    traffic = committed_traffic("apply_fine_fp32_cfg1.md")

    line = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_mx / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic: seeded uniform[0,1] densities (seed 1), r_min=1.5 filter",
        "config": {"workload": "192x96x96 hex8 cantilever, 5,447,811 dof, mixed "
                               "FP32/FP64 PCG + 5-level GMG to 1e-8",
                   "n_elem": ne, "n_dof": 3 * nn, "levels": cfg["levels"],
                   "l2": "working set > L2 (126 MB) per solve; apply timing flushes L2"},
        "iterations": info_mx[0]["iterations"], "outer": info_mx[0]["outer"],
        "relres": info_mx[0]["relres"], "compliance": info_mx[1],
        "fp64": {"value": round(value_64, 4), "unit": UNIT,
                 "ms_per_step": round(ms_64 / args.steps, 4),
                 "iterations": info_64[0]["iterations"],
                 "relres": info_64[0]["relres"], "compliance": info_64[1]},
        "mixed_over_fp64": round(value / value_64, 4),
        "setup_ms": round(setup_ms, 3),
        "setup_steady_ms": round(setup_steady_ms, 3),
        "setup_steady_fp64_ms": round(setup_steady_fp64, 3),
        "apply": {"fp32_ms": round(durs["fp32"], 5), "fp64_ms": round(durs["fp64"], 5),
                  "fp32_gbs": round(achieved32, 1), "fp64_gbs": round(achieved64, 1),
                  "bytes_fp32": bytes32, "bytes_fp64": bytes64},
        "roofline": {"bound": "hbm", "achieved": round(achieved32, 1),
                     "peak": peak, "unit": "GB/s",
                     "frac": round(achieved32 / peak, 4), "traffic": traffic,
                     "kernel": "k_apply_staged<float, 8, IN_U, OUT_Y>", "peak_kind": peak_kind},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    t.set_stream(None)
    # per-GPU figures of the other workloads: measured on one GPU only
    if not args.no_multi_rhs and world == 1:
        line["multi_rhs"] = run_multi_rhs(args, T, P, torch, dev, stream)
    if not args.no_buckling and world == 1:
        line["buckling"] = run_buckling(args, T, P, torch, dev, stream)
    if not args.no_oc and world == 1:
        line["oc_loop"] = run_oc_loop(args, T, P, torch, dev, stream)

    if not args.no_e2e:
        line["e2e"] = run_e2e(args, T, P, t, x, world, dev, torch)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline()
        Uo, Co, dco = cb.pop("_solution")
        line["cpu_baseline"] = cb
        # the acceptance check: both GPU forms against the FP64 oracle's
        # solution of the same problem (relative 2-norm errors)
        nrel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
        line["vs_oracle"] = {
            form: {"compliance_rel_err": abs(sol[1] - Co) / abs(Co),
                   "u_rel_err": nrel(sol[0], Uo), "dcdx_rel_err": nrel(sol[2], dco)}
            for form, sol in (("mixed", sol_mx), ("fp64", sol_64))}
        line["vs_oracle"]["oracle_iterations"] = cb["iterations"]
        line["compliance_rel_err_vs_oracle"] = line["vs_oracle"]["mixed"]["compliance_rel_err"]
    return line


def run_multi_rhs(args, T, P, torch, dev, stream, nrhs=8, reps=3):
    """Multi-load solves (128x64x64, `nrhs` seeded unit point loads on the
    x = 128 face): right-hand sides per second with blocks of 1, 4, 8 and
    the autotuned choice, mixed and FP64, device-resident loads."""
    cfg = "cfg2"
    c = P.CONFIGS[cfg]
    t = build_problem(T, P, cfg)
    t.set_stream(stream.cuda_stream)
    t.MatIntFnc(torch.tensor(P.design(cfg), device=dev))
    t.FEAssemble()
    F = torch.tensor(P.point_loads(c["nel"], nrhs, seed=2), device=dev)
    U = torch.zeros_like(F)
    out = {"workload": f"{c['nel'][0]}x{c['nel'][1]}x{c['nel'][2]} hex8, "
                       f"{3 * t.nNode} dof, {nrhs} point loads, 1e-8",
           "unit": "solves/s", "nrhs": nrhs, "reps": reps}
    for prec, pname in ((T.PREC_MIXED, "mixed"), (T.PREC_FP64, "fp64")):
        res = {}
        for block in (1, 4, 8, 0):
            opts = T.default_opts(precision=prec, rhs_block=block)
            times, its = [], 0
            for r in range(reps + 1):
                U.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                info = t.solve(F, U, nrhs=nrhs, opts=opts)
                e1.record(stream)
                torch.cuda.synchronize(dev)
                assert info["status"] == 0, info
                if r:                       # the first run is warm-up
                    times.append(e0.elapsed_time(e1))
                its = info["iterations"]
            ms = statistics.median(times)
            res["auto" if block == 0 else f"block{block}"] = {
                "value": round(nrhs / (ms / 1e3), 3), "ms": round(ms, 3),
                "iterations_sum": its}
        res["best_over_block1"] = round(
            max(v["value"] for k, v in res.items() if k != "block1")
            / res["block1"]["value"], 3)
        out[pname] = res
    t.set_stream(None)
    return out


def mma_pair(x, gv, dv):
    """Two constraints for the MMA timings: the volume constraint (value gv,
    gradient dv) and mean(x[:n/2]) <= 0.35, a linear constraint on the first
    half of the design variables.  Returns g (2) and dgdx (n x 2)."""
    n = x.size
    h = n // 2
    d2 = np.zeros(n)
    d2[:h] = 1.0 / h
    return np.array([gv, x[:h].mean() - 0.35]), np.stack([dv, d2], axis=1)


def run_oc_loop(args, T, P, torch, dev, stream, iters=50):
    """The optimisation loop of the 64x32x32 r=2 cantilever (Main.cpp:
    130-170): compliance objective, volume <= 0.3, 50 OC updates (51
    evaluations: MatIntFnc, FEAssemble, a warm-started mixed solve to 1e-8,
    C and V with gradients, OC update) through the Python API; and the OC
    update alone (the whole bisection in one persistent launch) and an MMA
    update with two constraints, on the final design."""
    cfg = "cfg3"
    c = P.CONFIGS[cfg]
    t = build_problem(T, P, cfg)
    t.set_stream(stream.cuda_stream)
    t.function_list = [T.Compliance([1.0], 0.0, 1.0, True, True),
                       T.Volume([0.3], 0.0, 1.0, False, True)]
    opts = T.default_opts(precision=T.PREC_MIXED)

    def loop():
        oc = T.OC(n=t.nElem, maxiter=iters)
        oc.xval = P.design(cfg)
        t.set("U", np.zeros(3 * t.nNode))
        return oc, T.optimize(t, oc, opts=opts)

    loop()                                  # warm-up (graphs, workspaces)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    oc, hist = loop()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    f, dfdx, g, dgdx = T.Function_Base.Function_Call(t)
    ups = []
    for r in range(11):
        oc2 = T.OC(n=t.nElem, maxiter=iters)
        oc2.xval = np.array(oc.xval)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        oc2.Update(t, dfdx, g, dgdx)
        b.record(stream)
        torch.cuda.synchronize(dev)
        if r:
            ups.append(a.elapsed_time(b))
    # MMA (m = 2: the volume constraint and mean(x) <= 0.35 over the first
    # half of the elements), one persistent launch per update: through the
    # Python class with host arrays, and through the C ABI with
    # device-resident state
    g2, dg2 = mma_pair(np.array(oc.xval), g[0], dgdx[:, 0])
    mups = []
    for r in range(11):
        mm = T.MMA(n=t.nElem, maxiter=iters)
        mm.xval = np.array(oc.xval)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        mm.Update(t, dfdx, g2, dg2)
        b.record(stream)
        torch.cuda.synchronize(dev)
        if r:
            mups.append(a.elapsed_time(b))
    import ctypes as C
    from topopt3d_b200 import _lib as L
    n = t.nElem
    xd = torch.tensor(np.array(oc.xval), device=dev)
    state = [xd.clone() for _ in range(3)] + [torch.zeros(n, device=dev, dtype=torch.float64),
                                              torch.ones(n, device=dev, dtype=torch.float64)]
    bounds = [torch.zeros(n, device=dev, dtype=torch.float64),
              torch.ones(n, device=dev, dtype=torch.float64)]
    dfd = torch.tensor(np.asarray(dfdx, np.float64), device=dev)
    dgd = torch.tensor(np.ascontiguousarray(dg2.T), device=dev)     # n x 2 column-major
    g2c = np.ascontiguousarray(g2, np.float64)
    mo = L.default_mma_opts()
    ch = C.c_double()
    ptr = lambda v: C.c_void_p(v.data_ptr())
    dups = []
    for r in range(11):
        for v, src in zip(state, [xd, xd, xd]):
            v.copy_(src)
        fresh = C.c_int32(1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rc = t._lib.tpo_mma_update(t._h, C.byref(mo), 0, C.byref(fresh), 2,
                                   *[ptr(v) for v in state], *[ptr(v) for v in bounds],
                                   ptr(dfd), g2c.ctypes.data_as(C.POINTER(C.c_double)),
                                   ptr(dgd), C.byref(ch), L.MEM_DEVICE)
        b.record(stream)
        torch.cuda.synchronize(dev)
        if rc != 0:
            raise RuntimeError(f"tpo_mma_update failed ({rc})")
        if r:
            dups.append(a.elapsed_time(b))
    nsteps = C.c_int32()
    t._lib.tpo_mma_last_info(t._h, C.byref(nsteps))
    t.set_stream(None)
    return {"workload": f"{c['nel'][0]}x{c['nel'][1]}x{c['nel'][2]} cantilever r=2, "
                        f"{t.nElem} elements, compliance + volume <= 0.3, "
                        f"{iters} OC updates, mixed solves to 1e-8",
            "unit": "ms", "ms": round(ms, 2), "evaluations": len(hist),
            "ms_per_iteration": round(ms / len(hist), 3),
            "pcg_iterations": int(sum(h["solve"]["iterations"] for h in hist)),
            "final_compliance": round(float(hist[-1]["values"][0]), 10),
            "oc_update_ms": round(statistics.median(ups), 3),
            "mma_update_m2_ms": round(statistics.median(mups), 3),
            "mma_update_m2_device_ms": round(statistics.median(dups), 3),
            "mma_newton_steps": int(nsteps.value)}


def run_buckling(args, T, P, torch, dev, stream, reps=2):
    """Linear buckling of the 96x48x48 column (698,691 dof): Ks from the
    FP64 solution and the 6 largest lambda of Ks phi = lambda K phi (block
    12, relative residual 1e-6), preconditioned by an FP64 or an FP32
    V-cycle.  Timed per call (Ks assembly + eigensolve) with CUDA events."""
    cfg = "cfg4"
    c = P.CONFIGS[cfg]
    t = build_problem(T, P, cfg)
    t.set_stream(stream.cuda_stream)
    t.MatIntFnc(torch.tensor(P.design(cfg), device=dev))
    o = T.default_opts(rtol=1e-12, maxit=5000)
    t.FEAssemble(o)
    t.FESolve(o)
    out = {"workload": f"{c['nel'][0]}x{c['nel'][1]}x{c['nel'][2]} column, "
                       f"{3 * t.nNode} dof, 6 largest lambda, block 12, tol 1e-6",
           "unit": "ms"}
    for pc, name in ((T.PREC_FP64, "fp64_vcycle"), (T.PREC_MIXED, "fp32_vcycle")):
        times = []
        for r in range(reps + 1):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            t.ks_assemble()
            lam = t.buckling(nev=6, block=12, precond=pc)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            if r:
                times.append(e0.elapsed_time(e1))
        out[name] = {"ms": round(statistics.median(times), 2),
                     "iterations": t.last_eig["iterations"],
                     "status": t.last_eig["status"],
                     "max_resid": t.last_eig["max_resid"],
                     "lambda": [round(float(v), 12) for v in lam]}
    # the design gradient of the aggregated value (Stability with
    # calc_gradient): 6 adjoint solves (mixed, blocks of right-hand sides),
    # the element kernels and the filter chain rule, device-resident
    lam, phi = t.buckling(nev=6, block=12, want_vectors=True)
    phi_d = torch.tensor(phi, device=dev)
    adj = T.default_opts(precision=T.PREC_MIXED)
    times = []
    for r in range(reps + 1):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        value, _ = t.buckling_sensitivity(lam, phi_d, opts=adj)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if r:
            times.append(e0.elapsed_time(e1))
    out["gradient"] = {"ms": round(statistics.median(times), 2),
                       "adjoint_iterations": t.last_adjoint["iterations"],
                       "status": t.last_adjoint["status"],
                       "value": round(value, 12)}
    # natural frequencies of the same column (Frequency, Dynamic.cpp:18-235):
    # lumped mass, more than 4 eigenpairs of M phi = lambda K phi (FP64
    # V-cycle preconditioner, tol 1e-6), value and design gradient
    times = []
    for r in range(reps + 1):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        lam_f, val_f, _ = t.frequency(4, 1.0, gradient=True)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if r:
            times.append(e0.elapsed_time(e1))
    out["frequency"] = {"ms": round(statistics.median(times), 2),
                        "pairs": int(lam_f.size),
                        "iterations": t.last_eig["iterations"],
                        "status": t.last_eig["status"],
                        "lambda": [round(float(v), 9) for v in lam_f]}
    t.set_stream(None)
    return out


def run_e2e(args, T, P, t, x, world, dev, torch):
    """Whole design iterations through the C ABI with host buffers: the
    design comes from pinned host memory and dC/dx goes back to it every
    step.  The displacement guess is reset to zero on the device (solver
    state, not an input), so every step does the work of a cold solve."""
    ne, nn = t.nElem, t.nNode
    x_h = torch.tensor(x, dtype=torch.float64).pin_memory()
    dc_h = torch.zeros(ne, dtype=torch.float64).pin_memory()
    u0 = torch.zeros(3 * nn, dtype=torch.float64, device=dev)
    mixed = T.default_opts(precision=T.PREC_MIXED)

    def step():
        t.MatIntFnc(x_h)                 # H2D of the design
        t.FEAssemble(mixed)
        t.set("U", u0)                   # cold start (device-side reset)
        t.FESolve(mixed)
        C, _, _ = t.compliance(out=dc_h)  # D2H of dC/dx (and C)
        return C

    for _ in range(args.warmup):
        step()
    barrier(world)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    t.FESolve  # noqa: B018 (keep the handle alive until timing ends)
    torch.cuda.synchronize(dev)
    el = max_over_ranks(time.perf_counter() - t0, world)
    return {"value": round(world * args.steps / el, 4), "unit": UNIT,
            "h2d_bytes_per_step": ne * 8,
            "d2h_bytes_per_step": ne * 8 + 8,
            "includes": "design upload, MatIntFnc, FEAssemble/PCSetUp, mixed solve, "
                        "compliance + dC/dx download"}


# ------------------------------------------------------------ CPU baseline

def cpu_baseline(steps=None, warmup=0, cfg=CONFIG):
    """The oracle's assembled FP64 PCG + GMG (OpenMP, all host threads) on
    the same problem (192x96x96 unless `cfg` names another).  Without
    `steps`: one complete solve from U = 0 is timed (solves/s = 1 / its
    time) and its solution is returned under "_solution".  With `steps`
    (the reference arm): `warmup` untimed and `steps` timed complete solves
    from U = 0; solves/s = 1 / their mean time."""
    from oracle import oracle as O
    from topopt3d_b200 import problems as P
    c = P.CONFIGS[cfg]
    cores = os.cpu_count()
    ref = O.Problem(c["nel"], rmin=c["rmin"], mg_levels=c["levels"])
    P.apply_bcs(ref, P.bcs(cfg))
    ref.set_design(P.design(cfg), 3.0, 1e-10)
    mesh = "x".join(str(v) for v in c["nel"])
    t0 = time.perf_counter()
    ref.assemble(O.default_opts())
    setup_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    U, st, its_full, rr = ref.solve(opts=O.default_opts())
    full_s = time.perf_counter() - t0
    if not steps:
        C, dc, _ = ref.compliance(U)
        return {"value": round(1.0 / full_s, 6), "unit": UNIT, "cores": cores,
                "kind": "port",
                "sample": f"one complete FP64 PCG+GMG solve from U=0 of the {mesh} "
                          f"problem ({its_full} iterations, relres {rr:.2e}, status {st}; "
                          f"assembled BSR SpMV, Galerkin PtAP, OpenMP); set-up "
                          f"{setup_s:.1f} s untimed",
                "full_solve_s": full_s, "setup_s": setup_s, "iterations": its_full,
                "_solution": (U, C, dc)}

    def full_solve():
        t0 = time.perf_counter()
        _, st_s, its_s, _ = ref.solve(opts=O.default_opts())
        if st_s != 0:
            raise RuntimeError(f"oracle solve failed: status {st_s}")
        return time.perf_counter() - t0, its_s

    for _ in range(warmup):
        full_solve()
    runs = [full_solve() for _ in range(steps)]
    mean_s = statistics.mean(r[0] for r in runs)
    return {"value": round(1.0 / mean_s, 6), "unit": UNIT, "cores": cores,
            "kind": "port",
            "sample": f"{steps} complete FP64 PCG+GMG solves from U=0 of the {mesh} "
                      f"problem ({its_full} iterations each; assembled BSR SpMV, "
                      f"Galerkin PtAP, OpenMP), mean time per solve; set-up "
                      f"{setup_s:.1f} s and {warmup + 1} warm-up solve(s) untimed",
            "solve_s": mean_s, "iterations": its_full}


def run_reference(args, rank, world):
    """Reference arm: the reference's FE path on the host cores.  The
    reference (PETSc/SLEPc/ParMETIS/MPI/Eigen) cannot be built in this image,
    so its CPU path runs as the oracle restatement."""
    if rank != 0:
        return None
    # the first complete solve (for the iteration count) is the warm-up
    cb = cpu_baseline(steps=args.steps, warmup=0, cfg=args.config)
    return {"impl": "reference", "metric": METRIC, "value": cb["value"],
            "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": ({"workload": "192x96x96 hex8 cantilever, 5,447,811 dof, FP64 "
                                    "PCG + 5-level GMG to 1e-8 (CPU)"}
                       if args.config == CONFIG else {"workload": args.config}),
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def run_kernel_case(args):
    """Profiling case: set up `args.config` and launch one operation
    `args.reps` times (the set-up launches precede them)."""
    import ctypes as C

    import torch

    import topopt3d_b200 as T
    from topopt3d_b200 import problems as P
    dev = torch.device("cuda", 0)
    t = build_problem(T, P, args.config)
    t.MatIntFnc(torch.tensor(P.design(args.config), device=dev))
    t.FEAssemble()
    torch.cuda.synchronize(dev)
    n = 3 * t.nNode
    lib = T.load()
    u64 = torch.randn(n, dtype=torch.float64, device=dev)
    y64 = torch.empty_like(u64)
    u32, y32 = u64.float(), torch.empty(n, dtype=torch.float32, device=dev)
    if args.kernel in ("level1_32", "level1_32_stencil"):
        # the FP32 level-1 operator: the tensor-core form or the stored stencil
        t.set_level1_form(1 if args.kernel == "level1_32_stencil" else 0)
        n1 = 3 * int(np.prod(t.level_dims(1)))
        u1 = torch.randn(n1, dtype=torch.float64, device=dev)
        y1 = torch.empty_like(u1)
    if args.kernel == "mma":
        # MMA update (m = 2, the constraints of mma_pair) at the design, with the
        # compliance sensitivity of one solve; device-resident state, reset
        # before each launch so every launch does the same work
        t.FESolve(T.default_opts())
        _, dC, _ = t.compliance(gradient=True)
        V, dV = t.volume(gradient=True)
        x0 = torch.tensor(P.design(args.config), device=dev)
        st = [x0.clone() for _ in range(3)] + [torch.zeros_like(x0), torch.ones_like(x0)]
        bnd = [torch.zeros_like(x0), torch.ones_like(x0)]
        dfd = torch.tensor(np.asarray(dC, np.float64), device=dev)
        g2, dg2 = mma_pair(P.design(args.config), V - 0.3, np.asarray(dV, np.float64))
        dgd = torch.tensor(np.ascontiguousarray(dg2.T), device=dev)
        from topopt3d_b200 import _lib as L
        mo = L.default_mma_opts()
        ch = C.c_double()
        ptr = lambda v: C.c_void_p(v.data_ptr())
    for _ in range(args.reps):
        if args.kernel == "mma":
            for v in st[:3]:
                v.copy_(x0)
            fresh = C.c_int32(1)
            rc = lib.tpo_mma_update(t._h, C.byref(mo), 0, C.byref(fresh), 2,
                                    *[ptr(v) for v in st], *[ptr(v) for v in bnd], ptr(dfd),
                                    g2.ctypes.data_as(C.POINTER(C.c_double)), ptr(dgd),
                                    C.byref(ch), L.MEM_DEVICE)
            assert rc == 0, lib.tpo_last_error(t._h)
            continue
        if args.kernel in ("setup", "setup_mixed"):
            # FEAssemble / PCSetUp for the same design: the whole hierarchy
            # (FP64 form, or the mixed form's FP32 Chebyshev bounds)
            t.FEAssemble(T.default_opts(precision=T.PREC_MIXED)
                         if args.kernel == "setup_mixed" else None)
            continue
        if args.kernel in ("level1_32", "level1_32_stencil"):
            t.apply_level(1, u1, y1, precision=T.PREC_MIXED)
            continue
        if args.kernel == "apply32":
            rc = lib.tpo_apply_f32(t._h, C.c_void_p(u32.data_ptr()),
                                   C.c_void_p(y32.data_ptr()))
            assert rc == 0, lib.tpo_last_error(t._h)
        elif args.kernel == "apply64":
            t.apply(u64, y64, precision=T.PREC_FP64)
        elif args.kernel in ("vcycle32", "vcycle64"):
            prec = T.PREC_MIXED if args.kernel == "vcycle32" else T.PREC_FP64
            t.vcycle(u64, y64, precision=prec)
        else:
            prec = T.PREC_MIXED if args.kernel == "solve_mixed" else T.PREC_FP64
            t.set("U", torch.zeros(n, dtype=torch.float64, device=dev))
            t.FESolve(T.default_opts(precision=prec, use_graph=0 if args.no_graph else 1))
    torch.cuda.synchronize(dev)
    extra = ""
    if args.kernel == "mma":
        steps = C.c_int32()
        lib.tpo_mma_last_info(t._h, C.byref(steps))
        extra = f" ({steps.value} dual Newton steps each)"
    print(f"{args.kernel} on {args.config}: {args.reps} launches done{extra}", flush=True)


def main():
    args = parse()
    if args.kernel:
        run_kernel_case(args)
        return
    rank, world, local = dist_setup(args)
    if args.impl == "reference":
        line = run_reference(args, rank, world)
    else:
        line = run_ours(args, rank, world, local)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
