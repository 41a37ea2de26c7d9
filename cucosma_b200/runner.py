"""Run cuCOSMA benchmark lists through this library.

    python -m cucosma_b200.runner LIST.csv [LIST.csv ...] [--out DIR] [--runs 100]
        [--warmup 3] [--precision native] [--rows 0:50:5] [--check] [--cublas]

Each LIST.csv uses the reference's TESTS_TO_RUN schema (one configuration per
row; the column order read by Kernel/cuda/run.sh:189: occupancy, TYPE,
VECTORTYPE2, VECTORTYPE4, M, N, K, the tile sizes, SPLIT_K, ALPHA, BETA,
SWIZZLE, A_OFFSET, B_OFFSET, ATOMIC_REDUCTION).  Every row runs as one GEMM
through the C ABI (cucosma_gemm) with the row's M, N, K, TYPE, ALPHA, BETA,
SPLIT_K and SWIZZLE (or, with --library-schedule, the library's own split-K
and swizzle); the tile and offset columns describe the reference
kernel's compile-time tiling and are recorded, not used (this library picks
its kernels at run time), and ATOMIC_REDUCTION is moot (the split-K reduction
here is always deterministic).

Timing follows the reference's benchmark mode (Kernel/cuda/src/benchmark.h):
warm-up calls, then RUNS timed calls, each preceded by a write of a buffer of
twice the L2 size so that every call starts with a cold L2, each call timed
with CUDA events.  The events measure GPU time, like the kernel durations of
the reference's nvprof traces: a bounded spin kernel (torch.cuda._sleep, about
0.25 ms) is queued ahead of the start event, so the host-side cost of issuing
the call (Python, argument set-up, launch) is hidden behind it and the interval
holds the call's kernels and the gaps between them.  With --cublas the same
protocol times torch.matmul (cuBLAS, TF32 off) on the same operands.

Output, per list, a directory <list>_<host>_<date>/ laid out like the
reference's archived runs so that its ResultReader scripts read it: for row
i a `config_<i>_<M>x<N>x<K>.csv` holding the row as config.h text and an
`nvprof_<i>_<M>x<N>x<K>.csv` trace in nvprof's CSV layout (three preamble
lines, header, units row, one line per timed call; cuBLAS lines first, this
library's lines named `cosmaSgemm[cucosma_b200 ...]`, Duration in us).  A
`results.csv` beside them summarises every row (median / min time, TFLOP/s,
and with --check the error against an FP64 product of sampled rows and
whether it is inside the rigorous error bound).
"""
from __future__ import annotations

import argparse
import csv
import datetime
import os
import socket
import sys

import numpy as np

import cucosma_b200 as cc

FIELDS = ["OCCUPANCY", "TYPE", "VECTORTYPE2", "VECTORTYPE4", "M", "N", "K", "THREADBLOCK_TILE_M",
          "THREADBLOCK_TILE_N", "THREADBLOCK_TILE_K", "LOAD_K", "WARP_TILE_M", "WARP_TILE_N", "THREAD_TILE_M",
          "THREAD_TILE_N", "SPLIT_K", "ALPHA", "BETA", "SWIZZLE", "A_OFFSET", "B_OFFSET", "ATOMIC_REDUCTION"]
L2_BYTES = 126 << 20
HIDE_CYCLES = 500_000  # spin queued ahead of each timed call: ~0.25 ms at 2 GHz, longer than issuing it


def gpu_time_us(call, flush):
    """GPU time of call() in us: cold L2, host issue hidden behind a spin."""
    import torch

    flush.zero_()
    torch.cuda._sleep(HIDE_CYCLES)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    call()
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1) * 1e3


def read_list(path):
    """Rows of a TESTS_TO_RUN file as dicts keyed by FIELDS (positional, so
    both header spellings of the first column work; header and blank lines
    skipped)."""
    rows = []
    with open(path, newline="") as f:
        for rec in csv.reader(f):
            rec = [x.strip() for x in rec]
            if len(rec) < len(FIELDS) or rec[4] in ("M", ""):
                continue
            rows.append(dict(zip(FIELDS, rec[:len(FIELDS)])))
    return rows


def config_text(row, when):
    """The row as the config.h text the reference generates (run.sh), line for
    line in the order its readers index (M on line 12, N 13, K 14 ...)."""
    lines = ["/*", " * config.h ", " *", " *  Created on: %s" % when, " *      Author: Automatically generated",
             " */", "#ifndef CONFIG_H_", "#define CONFIG_H_"]
    for key in ["TYPE", "VECTORTYPE2", "VECTORTYPE4", "M", "N", "K", "THREADBLOCK_TILE_M", "THREADBLOCK_TILE_N",
                "THREADBLOCK_TILE_K", "LOAD_K", "WARP_TILE_M", "WARP_TILE_N", "THREAD_TILE_M", "THREAD_TILE_N",
                "A_OFFSET", "B_OFFSET", "SWIZZLE", "SPLIT_K", "ATOMIC_REDUCTION"]:
        lines.append("#define %s %s" % (key, row[key]))
    lines.append("#define ADDITIONAL_OCCUPANCY_SM %s" % row["OCCUPANCY"])
    lines.append("#define ALPHA %s" % row["ALPHA"])
    lines.append("#define BETA %s" % row["BETA"])
    lines.append("#endif /* CONFIG_H_ */")
    return "\n".join(lines) + "\n"


NVPROF_HEADER = ('"Start","Duration","Grid X","Grid Y","Grid Z","Block X","Block Y","Block Z",'
                 '"Registers Per Thread","Static SMem","Dynamic SMem","Size","Throughput","SrcMemType","DstMemType",'
                 '"Device","Context","Stream","Name","Correlation_ID"')
NVPROF_UNITS = "s,us,,,,,,,,KB,KB,B,MB/s,,,,,,,"


def nvprof_text(device, entries):
    """entries: (start_s, duration_us, name) per timed call."""
    out = ["==0== NVPROF-compatible trace written by cucosma_b200.runner", "==0== Profiling application: cucosma_b200",
           "==0== Profiling result:", NVPROF_HEADER, NVPROF_UNITS]
    for i, (t0, dur, name) in enumerate(entries):
        out.append('%.6f,%.6f,,,,,,,,,,,,,,"%s","1","7","%s",%d' % (t0, dur, device, name, i))
    return "\n".join(out) + "\n"


def parse_rows(spec, n):
    if not spec:
        return range(n)
    parts = [int(p) if p else None for p in spec.split(":")]
    return range(n)[slice(*parts)]


def pitched(rows, cols, dtype, gen=None):
    """Device matrix with 16-byte aligned rows (like the reference callers'
    cudaMallocPitch): uniform[-1, 1] from gen, or zeros."""
    import torch

    es = torch.empty((), dtype=dtype).element_size()
    ld = max(1, -(-cols * es // 16)) * 16 // es
    if gen is None:
        buf = torch.zeros((max(rows, 1), ld), dtype=dtype, device="cuda")
    else:
        buf = torch.rand((max(rows, 1), ld), generator=gen, dtype=dtype, device="cuda") * 2 - 1
    return buf[:rows, :cols]


def run_row(row, args, flush, gen_seed):
    import torch

    dtype = torch.float64 if row["TYPE"] == "double" else torch.float32
    m, n, k = int(row["M"]), int(row["N"]), int(row["K"])
    alpha, beta = float(row["ALPHA"]), float(row["BETA"])
    split_k, swizzle = int(row["SPLIT_K"]), int(row["SWIZZLE"])
    es = 8 if dtype == torch.float64 else 4
    if (m * k + k * n + m * n) * es > args.max_gb * 1e9:
        return None, None, "skipped: operands exceed --max-gb"
    if (args.precision == "ozaki") != (dtype == torch.float64) and args.precision != "native":
        return None, None, "skipped: %s needs %s rows" % (args.precision, "double" if args.precision == "ozaki"
                                                            else "float")
    g = torch.Generator(device="cuda")
    g.manual_seed(gen_seed)
    A, B = pitched(m, k, dtype, g), pitched(k, n, dtype, g)
    C0 = pitched(m, n, dtype, g if beta != 0 else None)
    C = pitched(m, n, dtype)
    C.copy_(C0)
    prec = args.precision
    if args.library_schedule:
        split_k = swizzle = 0
    kw = dict(precision=prec, split_k=split_k if split_k > 1 else 0, swizzle=swizzle if swizzle > 1 else 0)
    desc = cc.make_desc(A, B, C, alpha, beta, **kw)
    ws = cc.alloc_workspace(desc)
    plan = cc.get_plan(desc)
    cc.gemm(A, B, C, alpha, beta, workspace=ws, **kw)
    check = None
    if args.check:
        torch.cuda.synchronize()
        idx = np.unique(np.linspace(0, m - 1, min(m, 8)).astype(np.int64))
        Ah = A[idx].double().cpu().numpy()
        Bh = B.double().cpu().numpy()
        Ch = C0[idx].double().cpu().numpy()
        ref = alpha * (Ah @ Bh) + beta * Ch
        u = 2.0 ** -53 if dtype == torch.float64 else 2.0 ** -24
        if prec in ("bf16x3", "bf16x6"):
            u_prod = 3.1 * 2.0 ** -16 if prec == "bf16x3" else 6 * 2.0 ** -24
            bnd = (u_prod + 6 * (k + 2) * 2.0 ** -24) * abs(alpha) * (np.abs(Ah) @ np.abs(Bh))
        else:
            bnd = (k + 2) * u * abs(alpha) * (np.abs(Ah) @ np.abs(Bh))
        bnd = 2 * (bnd + 2 * u * (np.abs(ref) + abs(beta) * np.abs(Ch))) + 1e-300
        out = C[torch.as_tensor(idx, device="cuda")].double().cpu().numpy()
        err = np.abs(out - ref)
        check = {"max_abs": float(err.max()), "normwise": float(np.linalg.norm(err) / max(np.linalg.norm(ref), 1e-300)),
                 "within_bound": bool(np.all(err <= bnd))}
    for _ in range(args.warmup):
        cc.gemm(A, B, C, alpha, beta, workspace=ws, **kw)
    entries = []
    ours = []
    name = "cosmaSgemm[cucosma_b200 %s %s]" % (prec, "splits=%d" % plan["splits"])
    if args.cublas:
        prev = torch.backends.cuda.matmul.allow_tf32
        torch.backends.cuda.matmul.allow_tf32 = False
        Ct = torch.empty((m, n), dtype=dtype, device="cuda")
        for _ in range(args.warmup):
            torch.matmul(A, B, out=Ct)
        for _ in range(args.runs):
            entries.append((0.0, gpu_time_us(lambda: torch.matmul(A, B, out=Ct), flush), "cublas[torch.matmul]"))
        torch.backends.cuda.matmul.allow_tf32 = prev
    for _ in range(args.runs):
        us = gpu_time_us(lambda: cc.gemm(A, B, C, alpha, beta, workspace=ws, **kw), flush)
        ours.append(us)
        entries.append((0.0, us, name))
    cub = [e[1] for e in entries if e[2].startswith("cublas")]
    res = {"M": m, "N": n, "K": k, "TYPE": row["TYPE"], "precision": prec, "splits": plan["splits"],
           "tile_m": plan["tile_m"], "tile_n": plan["tile_n"], "runs": args.runs,
           "median_us": float(np.median(ours)), "min_us": float(np.min(ours)),
           "tflops_median": 2.0 * m * n * k / (float(np.median(ours)) * 1e-6) / 1e12,
           "cublas_median_us": float(np.median(cub)) if cub else None}
    if check:
        res.update({"check_" + a: b for a, b in check.items()})
    return res, entries, None


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("lists", nargs="+", help="TESTS_TO_RUN-style CSV files")
    ap.add_argument("--out", default="cucosma_runs")
    ap.add_argument("--runs", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--precision", default="native", choices=["native", "bf16x3", "bf16x6", "ozaki"])
    ap.add_argument("--rows", default="", help="python slice of row indices, e.g. 0:512:8")
    ap.add_argument("--check", action="store_true", help="check each result on sampled rows against FP64")
    ap.add_argument("--cublas", action="store_true", help="also time torch.matmul (cuBLAS, TF32 off)")
    ap.add_argument("--max-gb", type=float, default=40.0, help="skip rows whose A + B + C exceed this")
    ap.add_argument("--library-schedule", action="store_true",
                    help="ignore the rows' SPLIT_K and SWIZZLE (tuned for the reference's GPU) and let the library choose")
    args = ap.parse_args(argv)

    import torch

    device = torch.cuda.get_device_name()
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")
    when = datetime.datetime.now().strftime("%a %b %d %H:%M:%S %Y")
    stamp = datetime.datetime.now().strftime("%Y-%m-%d_%H_%M_%S")
    failures = 0
    for path in args.lists:
        rows = read_list(path)
        d = os.path.join(args.out, "%s_%s_%s" % (os.path.basename(path), socket.gethostname(), stamp))
        os.makedirs(d, exist_ok=True)
        summary = []
        for i in parse_rows(args.rows, len(rows)):
            row = rows[i]
            tag = "%d_%sx%sx%s" % (i + 1, row["M"], row["N"], row["K"])
            res, entries, note = run_row(row, args, flush, 1000 + i)
            if res is None:
                summary.append({"row": i + 1, "M": row["M"], "N": row["N"], "K": row["K"], "note": note})
                continue
            with open(os.path.join(d, "config_%s.csv" % tag), "w") as f:
                f.write(config_text(row, when))
            with open(os.path.join(d, "nvprof_%s.csv" % tag), "w") as f:
                f.write(nvprof_text(device, entries))
            res["row"] = i + 1
            summary.append(res)
            if res.get("check_within_bound") is False:
                failures += 1
            print("%s row %d %sx%sx%s: median %.2f us, %.2f TFLOP/s%s" % (
                os.path.basename(path), i + 1, row["M"], row["N"], row["K"], res["median_us"], res["tflops_median"],
                "" if "check_within_bound" not in res else (", check %s" % ("ok" if res["check_within_bound"]
                                                                              else "FAILED"))), flush=True)
        keys = []
        for r in summary:
            keys += [k for k in r if k not in keys]
        with open(os.path.join(d, "results.csv"), "w", newline="") as f:
            w = csv.DictWriter(f, fieldnames=keys)
            w.writeheader()
            w.writerows(summary)
    st, code = cc.device_status()
    if st != cc.SUCCESS:
        print("device status %d (detail 0x%x)" % (st, code), file=sys.stderr)
        return 2
    return 1 if failures else 0


if __name__ == "__main__":
    sys.exit(main())
