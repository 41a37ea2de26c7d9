"""Benchmark of the cuCOSMA-compatible GEMM library on B200.

Workload (single GPU): the precision forms at M = N = K = 8192, alpha = 1,
beta = 0, entries i.i.d. uniform[-1, 1] from fixed seeds (synthetic; the
reference uses no dataset).  The headline "step" is one FP32 SGEMM through
the FP32-accurate BF16x6 tensor-core path (split pre-pass + CTA-pair tcgen05
GEMM), whose error against FP64 is at or below the native FP32 kernel's; the
same protocol times BF16x3 (faster, less accurate), the native FP32 (FFMA2)
SGEMM, the native FP64 (FP64 tensor-core MMA) DGEMM and the Ozaki INT8-slice
DGEMM (default call: 8 or 9 slices or native FP64, chosen on the device),
each reported with TFLOP/s, % of its relevant peak and its error against an
FP64 (double-double for FP64 paths) CPU oracle evaluated on a sample of rows.
results.spread repeats the forms on exponent-spread entries
sign * exp(N(0, 8^2)); results.families runs the reference's shape families
(square 8192^3, flat 16384^2 x 256, large-K 256^2 x 1,048,576, large-N
256 x 1,048,576 x 256) at alpha = 1, beta = 0.5, with and without the fused
sigmoid, through every path, with compute- and HBM-roofline fractions.

Timing: W untimed warm-up steps, then exactly K steps bracketed by a
barrier and torch.cuda.synchronize(), CUDA events on the launching stream,
max over ranks.  Every input is larger than the 126 MB L2 (256 MB per FP32
operand), so no flush is needed between steps.

cpu_baseline: the FP64 oracle (the reference's CPU product order,
Matrix.h:183-201) on a bounded sample of rows of the 8192^3 workload on all
host threads, plus the whole 1024^3 plain configuration single-threaded and
on all threads (cpu_baseline.p1024).

--impl reference times the reference's own CPU product
(Matrix<double>::operator*, Kernel/cuda/src/Matrix.h:183-201, built from its
sources into oracle/_ref/) on a bounded sample of rows of the same workload,
on all host threads.

Multi-GPU: the path does not shard (one GEMM per GPU); --gpus N runs N
independent replicas, one per rank, and reports the aggregate.

--precision-sweep (a separate mode beside the one-line benchmark) prints one JSON line per
(size, value distribution, path): sizes 8192 and 16384, entries uniform[-1, 1]
or sign * exp(N(0, sigma = 8)), paths native FP32, BF16x3, BF16x6, native FP64
and Ozaki with 6..9 slices; TFLOP/s and the max / mean relative and normwise
errors on 8 sampled rows against the FP64 (double-double for FP64 paths) oracle.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "TFLOP/s & % of peak: BF16x3/Ozaki vs native S/DGEMM at stated error vs FP64"
OZAKI_SLICES = 0  # the default call: 8 or 9 slices or native FP64, chosen on the device


def dram_traffic(path, n):
    """DRAM bytes (read + write) per launch of the path's main kernel at n^3, from
    the ncu capture recorded in profiles/dram_traffic.txt; None if not captured."""
    try:
        with open(os.path.join(ROOT, "profiles", "dram_traffic.txt")) as f:
            for line in f:
                t = line.split()
                if len(t) >= 5 and not t[0].startswith("#") and t[0] == path and t[1] == str(n):
                    return int(t[3]) + int(t[4])
    except (OSError, ValueError):
        pass
    return None


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return {"bf16": float(p["bf16_tflops"]), "bf16_sustained": float(p.get("bf16_tflops_sustained", 0) or 0),
                "hbm": float(p["hbm_gbs"]), "sm_max_mhz": float(p.get("sm_max_mhz", 1965.0)), "source": "measured"}
    except Exception:
        return {"bf16": 1590.0, "bf16_sustained": 1400.0, "hbm": 6650.0, "sm_max_mhz": 1965.0, "source": "fallback"}


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples (every 50 ms) of SM clock and throttle reasons."""

    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, loaded, mx, reasons = [], [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                clk, mx, pw = float(parts[0]), float(parts[1]), float(parts[2])
            except ValueError:
                continue
            sm.append(clk)
            if pw > 250.0:  # samples taken while a kernel was running
                loaded.append(clk)
                for nm, v in zip(names, parts[4:8]):
                    if v.lower() == "active":
                        reasons.add(nm)
        use = loaded or sm
        return {"sm_mhz": float(np.median(use)) if use else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "samples_under_load": len(loaded)}


# ------------------------------------------------------------ distributed
def dist_setup(n_gpus):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------- workload
def make_inputs(n, seed, dtype):
    import torch

    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    return torch.rand((n, n), generator=g, device="cuda", dtype=dtype) * 2 - 1


def time_path(cc, A, B, Cm, prec, slices, steps, warmup, world, workspace):
    """Average ms per call over exactly `steps` calls (device events), plus the
    main kernel's average ms and the library launch count in the timed region."""
    import torch

    kw = dict(precision=prec, slices=slices, workspace=workspace)
    for _ in range(warmup):
        cc.gemm(A, B, Cm, 1.0, 0.0, **kw)
    st = torch.cuda.current_stream()
    barrier(world)
    torch.cuda.synchronize()
    l0 = cc.launch_count()
    cc.profile_start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        cc.gemm(A, B, Cm, 1.0, 0.0, **kw)
    e1.record(st)
    barrier(world)
    torch.cuda.synchronize()
    kern_ms, kern_n = cc.profile_stop()
    launches = cc.launch_count() - l0
    ms = e0.elapsed_time(e1) / steps
    return ms, (kern_ms / kern_n if kern_n else None), launches


def e2e_path(cc, A_h, B_h, C_h, prec, slices, steps, warmup):
    """Same metric through the public host-buffer call (cucosma_gemm_host):
    every step copies A and B from pinned host memory and C back, inside the
    timed region; the library overlaps those copies with row-block GEMMs.
    The device buffer is allocated once, before timing."""
    import torch

    st = torch.cuda.current_stream()
    buf = cc.host_buffer(cc.host_desc(A_h, B_h, C_h, precision=prec, slices=slices))

    def one():
        cc.gemm_host(A_h, B_h, C_h, 1.0, 0.0, precision=prec, slices=slices, buffer=buf)

    for _ in range(warmup):
        one()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        one()
    e1.record(st)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def fwd_bwd_bench(cc, steps, warmup, n=4096, precision="bf16x3"):
    """Forward Y = sigmoid(A@B) and backward dA, dB (three GEMMs of n^3),
    A, B uniform[-0.1, 0.1], dY uniform[-1, 1]; one step = forward + backward."""
    import torch

    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    A = (torch.rand((n, n), generator=g, device="cuda") * 2 - 1) * 0.1
    B = (torch.rand((n, n), generator=g, device="cuda") * 2 - 1) * 0.1
    dY = torch.rand((n, n), generator=g, device="cuda") * 2 - 1
    Y, dA, dB = (torch.empty((n, n), device="cuda") for _ in range(3))
    ws_f = cc.alloc_workspace(cc.make_desc(A, B, Y, precision=precision, epilogue="sigmoid"))

    def step():
        cc.gemm(A, B, Y, 1.0, 0.0, precision=precision, epilogue="sigmoid", workspace=ws_f)
        cc.gemm_backward(A, B, Y, dY, dA, dB, precision=precision, epilogue="sigmoid")

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    return {"n": n, "precision": precision, "ms": ms, "tflops": 3 * 2.0 * n ** 3 / ms / 1e9,
            "what": "Y = sigmoid(A@B), dA = G@B^T, dB = A^T@G, G = dY*Y*(1-Y) fused"}


def grouped_shapes(count=512, seed=5):
    """512 GEMMs: M, N log-uniform in [64, 2048], K log-uniform in [64, 8192]."""
    r = np.random.default_rng(seed)
    lu = lambda a, b: int(np.exp(r.uniform(np.log(a), np.log(b))))  # noqa: E731
    return [(lu(64, 2048), lu(64, 2048), lu(64, 8192)) for _ in range(count)]


def grouped_bench(cc, precision, dtype, slices, steps, warmup, seed=5):
    """One persistent grouped launch (captured in a CUDA graph) against the
    same 512 problems as 512 separate calls of the single-problem path (also
    captured, so neither side pays Python launch overhead)."""
    import torch

    shapes = grouped_shapes(seed=seed)
    flop = sum(2.0 * m * n * k for m, n, k in shapes)
    es = torch.tensor([], dtype=dtype).element_size()
    al = 16 // es

    def rows(g, r, c):
        return (torch.rand((r, -(-c // al) * al), generator=g, device="cuda", dtype=dtype) * 2 - 1)[:, :c]

    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    probs = [(rows(g, m, k), rows(g, k, n), torch.zeros((m, -(-n // al) * al), device="cuda", dtype=dtype)[:, :n])
             for m, n, k in shapes]
    plan = cc.grouped(probs, precision=precision, slices=slices)
    ws_max = max(cc.workspace_size(cc.make_desc(A, B, Cm, precision=precision, slices=slices)) for A, B, Cm in probs)
    ws = torch.empty(max(ws_max, 256), dtype=torch.uint8, device="cuda")

    def separate(stream):
        for A, B, Cm in probs:
            cc.gemm(A, B, Cm, precision=precision, slices=slices, workspace=ws, stream=stream)

    plan()
    n0 = cc.launch_count()
    separate(None)
    torch.cuda.synchronize()
    launches_separate = cc.launch_count() - n0
    s = torch.cuda.Stream()
    g1, g2 = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g1, stream=s):
            plan(stream=s)
        with torch.cuda.graph(g2, stream=s):
            separate(s)

    def timed(graph):
        for _ in range(warmup):
            graph.replay()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            graph.replay()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    t_grp, t_sep = timed(g1), timed(g2)
    del g1, g2
    plan.close()
    return {"problems": len(shapes), "gflop": flop / 1e9, "grouped_ms": t_grp, "separate_ms": t_sep,
            "tflops": flop / (t_grp * 1e-3) / 1e12, "separate_tflops": flop / (t_sep * 1e-3) / 1e12,
            "speedup_vs_separate": t_sep / t_grp, "launches_grouped": 2 if precision != "ozaki" else 3,
            "launches_separate": launches_separate,
            "shapes": "M,N log-uniform [64,2048], K log-uniform [64,8192], seed %d" % seed}


# -------------------------------------------------------------- CPU legs
def make_dist(n, seed, dist):
    """FP64 device matrix: uniform[-1, 1], or sign * exp(X), X ~ N(0, 8^2)."""
    import torch

    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    if dist == "uniform":
        return torch.rand((n, n), generator=g, device="cuda", dtype=torch.float64) * 2 - 1
    sign = torch.where(torch.rand((n, n), generator=g, device="cuda", dtype=torch.float64) < 0.5, -1.0, 1.0)
    return sign * torch.exp(8.0 * torch.randn((n, n), generator=g, device="cuda", dtype=torch.float64))


def precision_sweep(args):
    """Precision forms at 8192^3 and 16384^3 on both value distributions."""
    import torch

    import cucosma_b200 as cc
    import oracle

    threads = oracle.lib().oracle_max_threads()
    sizes = [int(x) for x in args.sweep_sizes.split(",")]
    for n in sizes:
        for dist in ("uniform", "expspread"):
            A64, B64 = make_dist(n, 1, dist), make_dist(n, 2, dist)
            idx = np.linspace(0, n - 1, 8).astype(np.int64)
            A64h, B64h = A64.cpu().numpy(), B64.cpu().numpy()
            A32, B32 = A64.float(), B64.float()
            A32h, B32h = A32.cpu().numpy(), B32.cpu().numpy()
            ref32 = oracle.gemm(A32h[idx], B32h, threads=threads)
            hi, lo = oracle.gemm(A64h[idx], B64h, dd=True, threads=threads)
            del A64h, B64h, A32h, B32h
            paths = [("native_f32", "native", 0, A32, B32), ("bf16x3", "bf16x3", 0, A32, B32),
                     ("bf16x6", "bf16x6", 0, A32, B32), ("native_f64", "native", 0, A64, B64)]
            paths += [("ozaki_s%d" % s_, "ozaki", s_, A64, B64) for s_ in (6, 7, 8, 9)]
            for name, prec, slices, A, B in paths:
                Cm = torch.zeros((n, n), dtype=A.dtype, device="cuda")
                d = cc.make_desc(A, B, Cm, 1.0, 0.0, precision=prec, slices=slices)
                ws = cc.alloc_workspace(d)
                ms, kern_ms, _ = time_path(cc, A, B, Cm, prec, slices, args.steps, args.warmup, 1, ws)
                out = Cm[torch.as_tensor(idx, device="cuda")].cpu().numpy()
                err = oracle.errors(out, ref32) if A.dtype == torch.float32 else oracle.errors(out, hi, lo)
                err["nonfinite"] = int((~np.isfinite(out)).sum())
                print(json.dumps({"sweep": "precision", "n": n, "dist": dist, "path": name, "ms": ms,
                                  "tflops": 2.0 * n ** 3 / (ms * 1e-3) / 1e12, "kernel_ms": kern_ms,
                                  "error_vs_fp64": err}), flush=True)
                del Cm, ws
            del A64, B64, A32, B32
            torch.cuda.empty_cache()
    st, code = cc.device_status()
    if st != cc.SUCCESS:
        raise SystemExit("device status %d (detail 0x%x)" % (st, code))
    return 0


def cpu_sample(n, A32, B32, A64, B64, outs, budget_s=12.0):
    """CPU baseline leg: times the FP64 oracle on a bounded sample of rows of
    the FP32 workload (all host threads) and uses the same rows -- plus a
    double-double sample of the FP64 workload -- as the checker that states
    the error of each GPU result.  Returns (cpu_baseline, errors)."""
    import oracle

    threads = oracle.lib().oracle_max_threads()
    rows_probe = 8
    t0 = time.perf_counter()
    oracle.gemm(A32[:rows_probe], B32, threads=threads)
    dt = time.perf_counter() - t0
    rows = int(max(rows_probe, min(n, rows_probe * budget_s / max(dt, 1e-3))))
    rows = max(rows_probe, min(rows, 1024))
    idx = np.linspace(0, n - 1, rows).astype(np.int64)
    t0 = time.perf_counter()
    ref32 = oracle.gemm(A32[idx], B32, threads=threads)
    dt = time.perf_counter() - t0
    tflops = 2.0 * rows * n * n / dt / 1e12
    cpu = {"value": tflops, "unit": "TFLOP/s", "cores": threads, "kind": "port",
           "sample": "FP64 oracle (Matrix.h:183-201 order, OpenMP over rows) on %d of %d rows of the %d^3 FP32 "
                     "workload, %.1f s" % (rows, n, n, dt)}
    errs = {}
    for name, out in outs.items():
        if out is None:
            continue
        if out.dtype == np.float32:
            errs[name] = oracle.errors(out[idx], ref32)
    # FP64 paths: double-double reference on a few rows of the FP64 workload.
    r64 = np.linspace(0, n - 1, 8).astype(np.int64)
    hi, lo = oracle.gemm(A64[r64], B64, dd=True, threads=threads)
    for name, out in outs.items():
        if out is not None and out.dtype == np.float64:
            errs[name] = oracle.errors(out[r64], hi, lo)
    return cpu, errs


FAMILIES = [("SQ", 8192, 8192, 8192), ("FL", 16384, 16384, 256), ("LK", 256, 256, 1048576),
            ("LN", 256, 1048576, 256)]
FAMILY_PATHS = [("native_f32", "native", 4), ("bf16x3", "bf16x3", 4), ("bf16x6", "bf16x6", 4),
                ("native_f64", "native", 8), ("ozaki", "ozaki", 8)]


def families_bench(cc, pk, sms, steps, warmup, check_rows=4):
    """The reference's benchmark shape families (Benchmarks/TESTS_TO_RUN
    square / Flat / LargeK / LargeN) at the sizes the workload names, alpha = 1,
    beta = 0.5 with C uniform[-1, 1], without and with the fused sigmoid,
    through every path (Ozaki with its default, device-chosen slice count).
    Per entry: GPU time of one call (CUDA events over `steps` calls after
    `warmup`; every operand or C is larger than L2 except FL's 16 MB A and B),
    TFLOP/s, the fraction of the path's compute peak, the fraction of the
    HBM roofline for the algorithmic bytes sizeof(T) (MK + KN + 2MN), and the
    error on `check_rows` sampled rows of the first call's output against the
    FP64 oracle (FP32 paths) or the double-double oracle (FP64 paths)."""
    import torch

    import oracle

    out = {}
    hbm = pk["hbm"] * 1e9
    for fam, m, n, k in FAMILIES:
        flop = 2.0 * m * n * k
        for dt in (torch.float32, torch.float64):
            es = 4 if dt == torch.float32 else 8
            A = make_rect(m, k, 100, dt)
            B = make_rect(k, n, 101, dt)
            C0 = make_rect(m, n, 102, dt)
            rows = np.linspace(0, m - 1, check_rows).astype(np.int64)
            An, Bn, C0n = A[rows].double().cpu().numpy(), B.double().cpu().numpy(), C0[rows].double().cpu().numpy()
            refs = {}
            for name, prec, pes in FAMILY_PATHS:
                if pes != es:
                    continue
                for epi in ("none", "sigmoid"):
                    Cm = C0.clone()
                    d = cc.make_desc(A, B, Cm, 1.0, 0.5, precision=prec, epilogue=epi)
                    ws = cc.alloc_workspace(d)
                    plan = cc.get_plan(d)
                    cc.gemm(A, B, Cm, 1.0, 0.5, precision=prec, epilogue=epi, workspace=ws)
                    torch.cuda.synchronize()
                    first = Cm[rows].double().cpu().numpy()
                    choice = None
                    if prec == "ozaki" and plan["off_choice"]:
                        choice = int(ws[plan["off_choice"]: plan["off_choice"] + 4].view(torch.int32).item())
                    for _ in range(warmup):
                        cc.gemm(A, B, Cm, 1.0, 0.5, precision=prec, epilogue=epi, workspace=ws)
                    torch.cuda.synchronize()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    for _ in range(steps):
                        cc.gemm(A, B, Cm, 1.0, 0.5, precision=prec, epilogue=epi, workspace=ws)
                    e1.record()
                    torch.cuda.synchronize()
                    ms = e0.elapsed_time(e1) / steps
                    if epi not in refs:
                        code = oracle.EPI_SIGMOID if epi == "sigmoid" else oracle.EPI_NONE
                        refs[epi] = oracle.gemm(An, Bn, C0n, 1.0, 0.5, code, dd=(es == 8))
                    ref = refs[epi]
                    err = oracle.errors(first, *ref) if es == 8 else oracle.errors(first, ref)
                    peak = path_peak(name, pk, sms, choice if choice else 8)
                    algo = es * (m * k + k * n + 2 * m * n)
                    tf = flop / (ms * 1e-3) / 1e12
                    e = {"ms": ms, "tflops": tf, "compute_frac": tf / peak, "hbm_frac": algo / (ms * 1e-3) / hbm,
                         "algorithmic_bytes": algo, "normwise": err["normwise"], "max_abs": err["max_abs"],
                         "tile": [plan["tile_m"], plan["tile_n"]], "splits": plan["splits"]}
                    if choice is not None:
                        e["ozaki_choice"] = choice
                    out["%s_%s_%s" % (fam, name, epi)] = e
                    del ws, Cm
            del A, B, C0
            torch.cuda.empty_cache()
    out["inputs"] = "uniform[-1, 1], seeds 100 / 101 / 102 (A / B / C), alpha = 1, beta = 0.5"
    return out


def spread_bench(cc, n, pk, sms, steps, warmup, no_cpu=False, check_rows=4):
    """The precision forms on exponent-spread entries sign * exp(X), X ~ N(0,
    sigma = 8) at n^3 (alpha = 1, beta = 0): FP32 paths on the FP32 rounding
    of the FP64 values, FP64 paths on the values themselves (the default
    Ozaki call chooses its path on the device: reported as ozaki_choice).
    Time per call (CUDA events) and the error on sampled rows against the
    FP64 / double-double oracle."""
    import torch

    import oracle

    A64 = make_dist(n, 11, "spread")
    B64 = make_dist(n, 12, "spread")
    rows = np.linspace(0, n - 1, check_rows).astype(np.int64)
    flop = 2.0 * n ** 3
    res = {}
    ref = None
    for dt, names in ((torch.float32, ("native_f32", "bf16x3", "bf16x6")), (torch.float64, ("native_f64", "ozaki"))):
        A, B = (A64.float(), B64.float()) if dt == torch.float32 else (A64, B64)
        if not no_cpu:
            ref = oracle.gemm(A[rows].double().cpu().numpy(), B.double().cpu().numpy(), dd=(dt == torch.float64))
        for name in names:
            prec = "native" if name.startswith("native") else name
            Cm = torch.zeros((n, n), device="cuda", dtype=dt)
            d = cc.make_desc(A, B, Cm, precision=prec)
            ws = cc.alloc_workspace(d)
            plan = cc.get_plan(d)
            cc.gemm(A, B, Cm, precision=prec, workspace=ws)
            for _ in range(warmup):
                cc.gemm(A, B, Cm, precision=prec, workspace=ws)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(steps):
                cc.gemm(A, B, Cm, precision=prec, workspace=ws)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
            e = {"ms": ms, "tflops": flop / (ms * 1e-3) / 1e12}
            if name == "ozaki" and plan["off_choice"]:
                e["ozaki_choice"] = int(ws[plan["off_choice"]: plan["off_choice"] + 4].view(torch.int32).item())
            if ref is not None:
                o = Cm[rows].double().cpu().numpy()
                er = oracle.errors(o, *ref) if dt == torch.float64 else oracle.errors(o, ref)
                e["normwise"], e["mean_rel"] = er["normwise"], er["mean_rel"]
            res[name] = e
            del ws, Cm
        del A, B
    res["inputs"] = "sign * exp(N(0, 8^2)) per entry, %d^3, seeds 11 / 12" % n
    return res


def make_rect(rows, cols, seed, dtype):
    import torch

    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    return torch.rand((rows, cols), generator=g, device="cuda", dtype=dtype) * 2 - 1


def path_peak(name, pk, sms, slices):
    """Compute peak (TFLOP/s of useful flops) of a path."""
    if name == "native_f32":
        return sms * 128 * 2 * pk["sm_max_mhz"] * 1e6 / 1e12
    if name == "native_f64":
        return sms * 64 * 2 * pk["sm_max_mhz"] * 1e6 / 1e12
    if name == "bf16x3":
        return pk["bf16"] / 3
    if name == "bf16x6":
        return pk["bf16"] / 6
    return 2 * pk["bf16"] / (slices * (slices + 1) / 2)


def cpu_1024():
    """The reference-order FP64 product (Matrix.h:183-201, the oracle's
    restatement) on the whole 1024^3 problem of the plain configuration,
    single-threaded and on every host thread."""
    import oracle

    rng = np.random.default_rng(1)
    A = rng.uniform(-1, 1, (1024, 1024))
    B = rng.uniform(-1, 1, (1024, 1024))
    res = {}
    for label, th in (("single_thread", 1), ("all_threads", oracle.lib().oracle_max_threads())):
        t0 = time.perf_counter()
        oracle.gemm(A, B, threads=th)
        dt = time.perf_counter() - t0
        res[label] = {"threads": th, "s": dt, "tflops": 2.0 * 1024 ** 3 / dt / 1e12}
    try:
        model = [ln.split(":", 1)[1].strip() for ln in open("/proc/cpuinfo") if ln.startswith("model name")][0]
    except Exception:
        model = None
    res["cpu"] = model
    res["nproc"] = os.cpu_count()
    return res


def reference_arm(args):
    """--impl reference: the reference's own CPU product on host threads."""
    import ctypes as C
    from concurrent.futures import ThreadPoolExecutor

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    n = args.size
    import oracle

    rng = np.random.default_rng(1)
    threads = os.cpu_count() or 1
    rows_per_thread = max(1, args.ref_rows // threads)
    rows = rows_per_thread * threads
    B = rng.uniform(-1, 1, (n, n))
    A = rng.uniform(-1, 1, (rows, n))
    out = np.empty((rows, n))
    kind = "reference"
    if oracle.ref_available():
        L = oracle.ref_cpu()
        dp = C.POINTER(C.c_double)
        L.ref_cpu_set_b.argtypes = [C.c_int, C.c_int, dp]
        L.ref_cpu_rows.argtypes = [C.c_int, C.c_int, dp, dp]
        L.ref_cpu_set_b(n, n, B.ctypes.data_as(dp))

        def work(t):
            a = np.ascontiguousarray(A[t * rows_per_thread:(t + 1) * rows_per_thread])
            o = np.empty((rows_per_thread, n))
            L.ref_cpu_rows(rows_per_thread, n, a.ctypes.data_as(dp), o.ctypes.data_as(dp))
            out[t * rows_per_thread:(t + 1) * rows_per_thread] = o
    else:
        kind = "port"

        def work(t):
            sl = slice(t * rows_per_thread, (t + 1) * rows_per_thread)
            out[sl] = oracle.gemm(A[sl], B, threads=1)

    def step():
        with ThreadPoolExecutor(threads) as ex:
            list(ex.map(work, range(threads)))

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t0) / args.steps
    tflops = 2.0 * rows * n * n / dt / 1e12
    sample = ("Matrix<double>::operator* (Kernel/cuda/src/Matrix.h:183-201) on %d rows x %d x %d per step "
              "(%d threads x %d rows)" % (rows, n, n, threads, rows_per_thread))
    line = {"impl": "reference", "metric": METRIC, "value": tflops, "unit": "TFLOP/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "reference CPU product, sample of the %d^3 GEMM" % n, "m": n, "n": n, "k": n},
            "cpu_baseline": {"value": tflops, "unit": "TFLOP/s", "cores": threads, "kind": kind, "sample": sample},
            "e2e": {"value": tflops, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    gk = reference_gpu_kernel(n, args.steps, args.warmup)
    if gk:
        line["reference_gpu_kernel"] = gk
    print(json.dumps(line), flush=True)
    return 0


def reference_gpu_kernel(n, steps, warmup):
    """Informational: the reference kernel cosmaSgemm compiled unmodified for
    sm_100a from its sources (oracle/_ref, 8192^3, alpha 1, beta 0.5, tiles
    from its ScheduleGenerator) timed with CUDA events -- the plain FP32 kernel
    the precision paths are compared with.  Absent when not built or no GPU."""
    try:
        import torch

        import oracle

        tag = "f32_%d_a1b05" % n
        if not torch.cuda.is_available() or tag not in oracle.ref_kernel_tags():
            return None
        ref = oracle.RefKernel(tag)
        ld = -(-n // 128) * 128  # cudaMallocPitch-like rows
        g = torch.Generator(device="cuda")
        g.manual_seed(1)
        A = (torch.rand((n, ld), generator=g, device="cuda") * 2 - 1)
        B = (torch.rand((n, ld), generator=g, device="cuda") * 2 - 1)
        C = torch.zeros((n, ld), device="cuda")
        for _ in range(max(1, warmup)):
            ref(A.data_ptr(), ld, B.data_ptr(), ld, C.data_ptr(), ld)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            ref(A.data_ptr(), ld, B.data_ptr(), ld, C.data_ptr(), ld)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        return {"what": "cosmaSgemm (cuCOSMAV100.cuh) built for sm_100a, %d^3 FP32 SIMT, config %s" % (n, ref.config),
                "ms": ms, "tflops": 2.0 * n ** 3 / ms / 1e9}
    except Exception as e:  # informational only
        return {"error": str(e)[:200]}


# -------------------------------------------------------------------- main
def shape_run(args):
    """One GEMM shape through the library's default plan (--shape M,N,K), for
    profiling: W warm-up and K timed calls on uniform[-1, 1] inputs, CUDA
    events on the current stream; prints the plan and the time per call."""
    import torch

    import cucosma_b200 as cc

    m, n, k = (int(x) for x in args.shape.split(","))
    dt = torch.float64 if args.precision == "ozaki" or args.precision == "native_f64" else torch.float32
    prec = "native" if args.precision.startswith("native") else args.precision
    A = make_rect(m, k, 100, dt)
    B = make_rect(k, n, 101, dt)
    C = make_rect(m, n, 102, dt)
    d = cc.make_desc(A, B, C, 1.0, args.beta, precision=prec, epilogue=args.epilogue, tile=args.tile,
                     swizzle=args.swizzle)
    ws = cc.alloc_workspace(d)

    def call():
        cc.gemm(A, B, C, 1.0, args.beta, precision=prec, epilogue=args.epilogue, workspace=ws, tile=args.tile,
                swizzle=args.swizzle)

    for _ in range(args.warmup):
        call()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        call()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    es = 4 if dt == torch.float32 else 8
    gb = es * (m * k + k * n + (2 if args.beta else 1) * m * n) / 1e9
    print(json.dumps({"shape": [m, n, k], "precision": args.precision, "beta": args.beta, "epilogue": args.epilogue,
                      "ms": ms, "tflops": 2.0 * m * n * k / ms / 1e9, "algorithmic_tb_s": gb / ms,
                      "plan": cc.get_plan(d)}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=8192)
    ap.add_argument("--ref-rows", type=int, default=32)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline / error leg")
    ap.add_argument("--only", default="", help="comma-separated subset of paths (profiling runs): "
                    "bf16x3,bf16x6,native_f32,ozaki,native_f64,grouped_bf16x3,grouped_ozaki,fwd_bwd")
    ap.add_argument("--precision-sweep", action="store_true", help="precision forms x sizes x distributions")
    ap.add_argument("--sweep-sizes", default="8192,16384")
    ap.add_argument("--no-families", action="store_true", help="skip the reference shape families")
    ap.add_argument("--family-steps", type=int, default=3)
    ap.add_argument("--shape", default="", help="M,N,K: time one GEMM of this shape (profiling runs; with "
                    "--precision, --beta, --epilogue) and print its plan and time instead of the bench line")
    ap.add_argument("--precision", default="bf16x3")
    ap.add_argument("--beta", type=float, default=0.5)
    ap.add_argument("--epilogue", default="none")
    ap.add_argument("--tile", type=int, default=0, help="with --shape: tile id (0: the library's choice)")
    ap.add_argument("--swizzle", type=int, default=0, help="with --shape: raster band (0: the library's choice)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return reference_arm(args)
    if args.precision_sweep:
        return precision_sweep(args)
    if args.shape:
        return shape_run(args)

    import torch

    import cucosma_b200 as cc

    world, rank, local = dist_setup(args.gpus)
    n = args.size
    pk = peaks()
    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    sms = props.multi_processor_count

    A32 = make_inputs(n, 1 + 10 * rank, torch.float32)
    B32 = make_inputs(n, 2 + 10 * rank, torch.float32)
    C32 = torch.zeros((n, n), dtype=torch.float32, device="cuda")
    A64 = make_inputs(n, 3 + 10 * rank, torch.float64)
    B64 = make_inputs(n, 4 + 10 * rank, torch.float64)
    C64 = torch.zeros((n, n), dtype=torch.float64, device="cuda")

    paths = [("bf16x3", A32, B32, C32, 0), ("bf16x6", A32, B32, C32, 0), ("native_f32", A32, B32, C32, 0),
             ("ozaki", A64, B64, C64, OZAKI_SLICES), ("native_f64", A64, B64, C64, 0)]
    if args.only:
        keep = set(args.only.split(","))
        paths = [p for p in paths if p[0] in keep]
    flop = 2.0 * n * n * n
    results, outs = {}, {}
    # Clocks are sampled across all timed regions of this run (the headline
    # region alone is tens of milliseconds, shorter than the sampling period).
    sampler = ClockSampler(local)
    sampler.start()
    peak_names = {"native_f32": "FP32 SIMT (SMs x 128 x 2 x max clock)", "native_f64": "FP64 (SMs x 64 x 2 x max clock)",
                  "bf16x3": "measured bf16 dense / 3 products", "bf16x6": "measured bf16 dense / 6 products"}
    for name, A, B, Cm, slices in paths:
        prec = "native" if name.startswith("native") else name
        d = cc.make_desc(A, B, Cm, 1.0, 0.0, precision=prec, slices=slices)
        try:
            ws = cc.alloc_workspace(d)
            cc.gemm(A, B, Cm, 1.0, 0.0, precision=prec, slices=slices, workspace=ws)
        except cc.CucosmaError as e:
            if e.status == cc.NOT_SUPPORTED:
                results[name] = {"available": False}
                continue
            raise
        plan = cc.get_plan(d)
        choice = None
        if name == "ozaki":
            torch.cuda.synchronize()
            choice = (int(ws[plan["off_choice"]: plan["off_choice"] + 4].view(torch.int32).item())
                      if plan["off_choice"] else slices)
        ms, kern_ms, launches = time_path(cc, A, B, Cm, prec, slices, args.steps, args.warmup, world, ws)
        ms = max_over_ranks(ms, world)
        tf = flop / (ms * 1e-3) / 1e12
        if name == "ozaki":
            sl = choice if choice else 8
            peak = path_peak(name, pk, sms, sl)
            peak_name = "INT8 dense (2 x measured bf16) / %d slice products" % (sl * (sl + 1) // 2)
        else:
            peak, peak_name = path_peak(name, pk, sms, 0), peak_names[name]
        results[name] = {"available": True, "ms": ms, "tflops": tf, "pct_of_peak": 100.0 * tf / peak,
                         "peak_tflops": peak, "peak": peak_name, "kernel_ms": kern_ms, "launches_per_step":
                         launches / args.steps, "workspace_bytes": (ws.numel() if ws is not None else 0),
                         "tile": [plan["tile_m"], plan["tile_n"]]}
        if kern_ms:
            results[name]["kernel_frac"] = flop / (kern_ms * 1e-3) / 1e12 / peak
        if choice is not None:
            results[name]["ozaki_choice"] = choice
        outs[name] = Cm.cpu().numpy().copy() if rank == 0 and not args.no_cpu else None

    for gname, gprec, gdt, gsl in (("grouped_bf16x3", "bf16x3", torch.float32, 0),
                                   ("grouped_ozaki", "ozaki", torch.float64, OZAKI_SLICES)):
        if not args.only or gname in args.only.split(","):
            results[gname] = grouped_bench(cc, gprec, gdt, gsl, max(3, args.steps), args.warmup, seed=5 + 10 * rank)
    if not args.only or "fwd_bwd" in args.only.split(","):
        results["fwd_bwd_bf16x3"] = fwd_bwd_bench(cc, max(3, args.steps), args.warmup)
        results["fwd_bwd_bf16x6"] = fwd_bwd_bench(cc, max(3, args.steps), args.warmup, precision="bf16x6")
    if (not args.only or "spread" in args.only.split(",")) and rank == 0:
        results["spread"] = spread_bench(cc, n, pk, sms, max(2, args.family_steps), 1, no_cpu=args.no_cpu)
    if (not args.only and not args.no_families) or "families" in args.only.split(","):
        results["families"] = families_bench(cc, pk, sms, args.family_steps, 1)
    avail = [p for p in paths if results.get(p[0], {}).get("available")]
    if not avail:  # a profiling run of the grouped launches only
        clocks = sampler.stop()
        if rank == 0:
            print(json.dumps({"metric": METRIC, "results": results, "clocks": clocks}), flush=True)
        return 0
    # Headline: the FP32-accurate tensor-core form (BF16x6: error at or below
    # native FP32's); BF16x3 is reported beside it with its larger error.
    head_path = next((p for p in avail if p[0] == "bf16x6"), avail[0])
    head, hA, hB, hC, hslices = head_path
    hprec = "native" if head.startswith("native") else head
    hr = results[head]
    A_h = hA.cpu().pin_memory()
    B_h = hB.cpu().pin_memory()
    C_h = torch.empty_like(hC, device="cpu").pin_memory()
    e2e_ms = e2e_path(cc, A_h, B_h, C_h, hprec, hslices, max(3, args.steps // 2), 3)
    e2e_ms = max_over_ranks(e2e_ms, world)
    clocks = sampler.stop()
    es = hC.element_size()

    cpu, errs = (None, {})
    if rank == 0 and not args.no_cpu:
        cpu, errs = cpu_sample(n, A32.cpu().numpy(), B32.cpu().numpy(), A64.cpu().numpy(), B64.cpu().numpy(), outs)
        for name, e in errs.items():
            results[name]["error_vs_fp64"] = e
        cpu["p1024"] = cpu_1024()

    # roofline of the headline's main kernel (useful flops / kernel time)
    kern_ms = hr.get("kernel_ms") or hr["ms"]
    achieved = flop / (kern_ms * 1e-3) / 1e12
    roof = {"bound": "tensor" if not head.startswith("native") else "simt", "achieved": achieved,
            "peak": hr["peak_tflops"], "unit": "TFLOP/s", "frac": achieved / hr["peak_tflops"],
            "traffic": dram_traffic(head, n),
            "peak_source": pk["source"] + ": " + hr["peak"], "kernel_ms": kern_ms}
    dtypes = {"bf16x3": "bf16x3->f32", "bf16x6": "bf16x6->f32", "native_f32": "f32", "ozaki": "i8->f64",
              "native_f64": "f64"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": hr["tflops"] * world, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": hr["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": dtypes[head], "data": "synthetic",
            "config": {"workload": "GEMM %s %d^3, alpha=1 beta=0, U[-1,1]" % (head, n), "m": n, "n": n, "k": n,
                       "parallelism": "replicas" if world > 1 else "single-gpu",
                       "l2": "inputs larger than L2 (%d MB per operand), no flush" % (n * n * es >> 20)},
            "e2e": {"value": flop / (e2e_ms * 1e-3) / 1e12 * world, "unit": "TFLOP/s",
                    "h2d_bytes_per_step": 2 * n * n * es, "d2h_bytes_per_step": n * n * es},
            "gpu_launches": int(hr["launches_per_step"] * args.steps),
            "roofline": roof, "cpu_baseline": cpu, "clocks": clocks, "results": results,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
