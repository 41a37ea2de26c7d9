"""Shared helpers for the parity tests: seeded inputs, pitched device copies
and the rigorous error bound the FP32/FP64 results are held to."""
from __future__ import annotations

import numpy as np

import oracle

U32 = 2.0 ** -24
U64 = 2.0 ** -53


def uniform(seed, shape, dtype=np.float32, lo=-1.0, hi=1.0):
    return np.random.default_rng(seed).uniform(lo, hi, shape).astype(dtype)


def expspread(seed, shape, sigma=8.0, dtype=np.float64):
    """sign * exp(N(0, sigma)) per entry: exponents spread over ~2^+-35."""
    r = np.random.default_rng(seed)
    return (np.where(r.random(shape) < 0.5, -1.0, 1.0) * np.exp(r.normal(0.0, sigma, shape))).astype(dtype)


def to_dev(x, ld=None, device="cuda"):
    """Copy a 2-D numpy array into a row-major device buffer with row stride
    ld (elements, default: rounded up to 16 bytes) and return the view."""
    import torch

    x = np.ascontiguousarray(x)
    rows, cols = x.shape
    es = x.dtype.itemsize
    if ld is None:
        ld = -(-cols * es // 16) * 16 // es
        ld = max(ld, 16 // es)
    t = torch.zeros((max(rows, 1), ld), dtype=getattr(torch, str(x.dtype)), device=device)
    v = t[:rows, :cols]
    v.copy_(torch.from_numpy(x))
    return v


def bound(A, B, Cin, alpha, beta, epilogue, dtype, ref_pre):
    """Componentwise worst-case error bound of alpha*A@B + beta*C computed in
    floating point of the given dtype with any summation order:
      |err| <= gamma_{k+2} |alpha| (|A||B|) + 2u |beta C| + 2u |result|,
    then the sigmoid (1/4-Lipschitz) or ReLU (1-Lipschitz) epilogue."""
    u = U32 if dtype == np.float32 else U64
    k = A.shape[1]
    absab = oracle.gemm(np.abs(A), np.abs(B)) if k > 0 else np.zeros((A.shape[0], B.shape[1]))
    g = (k + 2) * u / (1 - (k + 2) * u)
    b = g * abs(alpha) * absab + 2 * u * np.abs(ref_pre)
    if beta != 0 and Cin is not None:
        b = b + 2 * u * abs(beta) * np.abs(np.asarray(Cin, np.float64))
    if epilogue == oracle.EPI_SIGMOID:
        b = 0.25 * b + 8 * u
    b = b + 1e-300
    return b


def check_against_oracle(out, A, B, Cin, alpha, beta, epilogue, dtype, factor=1.0):
    """Asserts out is within the rigorous bound of the FP64 oracle; returns the errors."""
    pre = oracle.gemm(A, B, Cin, alpha, beta, oracle.EPI_NONE)
    ref = oracle.gemm(A, B, Cin, alpha, beta, epilogue) if epilogue != oracle.EPI_NONE else pre
    b = bound(A, B, Cin, alpha, beta, epilogue, dtype, pre) * factor
    out = np.asarray(out, np.float64)
    err = np.abs(out - ref)
    bad = err > b
    if bad.any():
        i = np.argwhere(bad)[0]
        raise AssertionError("%d of %d entries outside the bound; first at %s: out=%r ref=%r err=%.3e bound=%.3e"
                             % (bad.sum(), bad.size, tuple(i), out[tuple(i)], ref[tuple(i)], err[tuple(i)], b[tuple(i)]))
    return oracle.errors(out, ref)


def bf16_bound(A, B, Cin, alpha, beta, nterms):
    """|err| <= (c_split + 6 (k+2) u32) |alpha| (|A||B|) + 2 u32 |beta C| + 2 u32 |result|,
    c_split = 3.1 * 2^-16 for BF16x3 (dropped lo*lo and the two residuals),
    6 * 2^-24 for BF16x6."""
    k = A.shape[1]
    u = 2.0 ** -24
    c_split = 3.1 * 2.0 ** -16 if nterms == 2 else 6.0 * u
    absab = oracle.gemm(np.abs(A), np.abs(B))
    ref = oracle.gemm(A, B, Cin, alpha, beta)
    b = (c_split + 6 * (k + 2) * u) * abs(alpha) * absab + 2 * u * np.abs(ref) + 1e-30
    if beta:
        b += 2 * u * abs(beta) * np.abs(Cin.astype(np.float64))
    return ref, b
