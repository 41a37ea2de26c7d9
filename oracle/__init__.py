"""CPU oracle for the cuCOSMA GEMM path.  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package.  The product (cucosma_b200) never does: it is the checker, not
the thing measured or shipped.

Contents
  liboracle.so (oracle.c)   FP64 / double-double GEMM restatement of
                            Matrix<T>::operator* (Kernel/cuda/src/Matrix.h:183-201)
                            with the alpha/beta epilogue of cuCOSMAV100.cuh:1582-1593,
                            BF16 split and Ozaki slice restatements.
  _ref/                     the reference's own code compiled from its sources
                            (oracle/build_ref.py): CPU product, input generator,
                            ScheduleGenerator, and the cosmaSgemm kernel per config.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

EPI_NONE, EPI_SIGMOID, EPI_RELU = 0, 1, 2

_lib = None


def build():
    """Compile liboracle.so (and oracle/_ref when the reference sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    from . import build_ref

    build_ref.build(verbose=False)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        L = C.CDLL(path)
        i64, dp, fp, i32p, i8p = C.c_int64, C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_int32), C.POINTER(C.c_int8)
        L.oracle_gemm_f64.argtypes = [i64, i64, i64, dp, i64, dp, i64, dp, i64, C.c_double, C.c_double, C.c_int, dp, i64, C.c_int]
        L.oracle_gemm_dd.argtypes = [i64, i64, i64, dp, i64, dp, i64, dp, i64, C.c_double, C.c_double, C.c_int, dp, i64, dp, C.c_int]
        L.oracle_splitk_reduce_f32.argtypes = [i64, i64, C.c_int, fp, fp, i64, C.c_float, C.c_float]
        L.oracle_split_bf16.argtypes = [fp, i64, C.c_int, C.POINTER(C.c_uint16)]
        L.oracle_ozaki_exponents.argtypes = [i64, i64, i64, dp, i64, dp, i64, i32p, i32p]
        L.oracle_ozaki_slices.argtypes = [i64, i64, i64, dp, i64, dp, i64, i32p, i32p, C.c_int, i8p, i8p]
        L.oracle_ozaki_gemm.argtypes = [i64, i64, i64, i8p, i8p, i32p, i32p, C.c_int, i64, dp, i64, C.c_double, C.c_double, C.c_int, dp, i64, C.c_int]
        L.oracle_max_threads.restype = C.c_int
        _lib = L
    return _lib


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def _f64(x):
    return np.ascontiguousarray(x, dtype=np.float64)


def gemm(A, B, Cin=None, alpha=1.0, beta=0.0, epilogue=EPI_NONE, dd=False, threads=0):
    """alpha*A@B + beta*C (then the epilogue) with FP64 (or double-double) dots.

    A: (m,k), B: (k,n), C: (m,n); any float dtype (converted exactly to FP64).
    Returns FP64 (m,n); with dd=True returns (hi, lo)."""
    A, B = _f64(A), _f64(B)
    m, k = A.shape
    k2, n = B.shape
    assert k == k2
    Cp = _f64(Cin) if Cin is not None else np.zeros((1, 1))
    out = np.empty((m, n), dtype=np.float64)
    ldc = Cp.shape[1] if Cin is not None else 0
    if dd:
        lo = np.empty_like(out)
        lib().oracle_gemm_dd(m, n, k, _p(A, C.c_double), k, _p(B, C.c_double), n, _p(Cp, C.c_double), ldc,
                             alpha, beta, epilogue, _p(out, C.c_double), n, _p(lo, C.c_double), threads)
        return out, lo
    lib().oracle_gemm_f64(m, n, k, _p(A, C.c_double), k, _p(B, C.c_double), n, _p(Cp, C.c_double), ldc,
                          alpha, beta, epilogue, _p(out, C.c_double), n, threads)
    return out


def splitk_reduce_f32(ws, Cin, alpha, beta):
    ws = np.ascontiguousarray(ws, dtype=np.float32)
    s, m, n = ws.shape
    Cout = np.array(Cin, dtype=np.float32, copy=True, order="C")
    lib().oracle_splitk_reduce_f32(m, n, s, _p(ws, C.c_float), _p(Cout, C.c_float), n, alpha, beta)
    return Cout


def split_bf16(x, nterms):
    """BF16 terms (uint16 bit patterns), shape (nterms,) + x.shape."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty((nterms,) + x.shape, dtype=np.uint16)
    lib().oracle_split_bf16(_p(x, C.c_float), x.size, nterms, _p(out, C.c_uint16))
    return out


def bf16_to_f32(h):
    return (np.asarray(h, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32)


def ozaki_exponents(A, B):
    A, B = _f64(A), _f64(B)
    m, k = A.shape
    n = B.shape[1]
    ea = np.empty(m, np.int32)
    eb = np.empty(n, np.int32)
    lib().oracle_ozaki_exponents(m, n, k, _p(A, C.c_double), k, _p(B, C.c_double), n, _p(ea, C.c_int32), _p(eb, C.c_int32))
    return ea, eb


def ozaki_slices(A, B, s):
    """(ea, eb, sa[s,m,k], sb[s,n,k]) int8 slices, B stored transposed."""
    A, B = _f64(A), _f64(B)
    m, k = A.shape
    n = B.shape[1]
    ea, eb = ozaki_exponents(A, B)
    sa = np.empty((s, m, k), np.int8)
    sb = np.empty((s, n, k), np.int8)
    lib().oracle_ozaki_slices(m, n, k, _p(A, C.c_double), k, _p(B, C.c_double), n, _p(ea, C.c_int32), _p(eb, C.c_int32),
                              s, _p(sa, C.c_int8), _p(sb, C.c_int8))
    return ea, eb, sa, sb


def ozaki_magnitude_sums(A, B):
    """Fixed-point magnitude sums of the adaptive Ozaki path: per row i of A,
    sum_k floor(|a_ik| 2^(30 - ea_i)); per column j of B the same with eb_j
    (ea, eb the Ozaki exponents).  Exact integers (Python ints)."""
    A, B = _f64(A), _f64(B)
    ea, eb = ozaki_exponents(A, B)
    ra = np.floor(np.ldexp(np.abs(A), (30 - ea.astype(np.int64))[:, None])).astype(np.uint64)
    rb = np.floor(np.ldexp(np.abs(B), (30 - eb.astype(np.int64))[None, :])).astype(np.uint64)
    return [int(x) for x in ra.sum(axis=1, dtype=np.uint64)], [int(x) for x in rb.sum(axis=0, dtype=np.uint64)]


def ozaki_choice(A, B):
    """Restatement of the device's path choice for the default Ozaki call
    (ozaki_choice in cucosma_b200/csrc/split.cuh): with P = K 2^30 / min
    nonzero row sum and Q = K 2^30 / min nonzero column sum, the smallest s in
    {8, 9} with 7 s >= 53 + log2(P + Q), else 0 (native FP64); 8 when A or B
    is all zero."""
    k = np.asarray(A).shape[1]
    sa, sb = ozaki_magnitude_sums(A, B)
    nza, nzb = [x for x in sa if x], [x for x in sb if x]
    if not nza or not nzb:
        return 8
    P = k * 1073741824.0 / float(min(nza))
    Q = k * 1073741824.0 / float(min(nzb))
    need = 53.0 + np.log2(P + Q)
    for s in (8, 9):
        if 7.0 * s >= need:
            return s
    return 0


def ozaki_gemm(A, B, s, Cin=None, alpha=1.0, beta=0.0, epilogue=EPI_NONE, kchunk=0, threads=0):
    """Bit-exact restatement of the Ozaki INT8-slice DGEMM (see oracle.c)."""
    A, B = _f64(A), _f64(B)
    m, k = A.shape
    n = B.shape[1]
    ea, eb, sa, sb = ozaki_slices(A, B, s)
    Cp = _f64(Cin) if Cin is not None else np.zeros((1, 1))
    ldc = Cp.shape[1] if Cin is not None else 0
    out = np.empty((m, n), np.float64)
    lib().oracle_ozaki_gemm(m, n, k, _p(sa, C.c_int8), _p(sb, C.c_int8), _p(ea, C.c_int32), _p(eb, C.c_int32), s, kchunk,
                            _p(Cp, C.c_double), ldc, alpha, beta, epilogue, _p(out, C.c_double), n, threads)
    return out


def errors(x, ref, ref_lo=None):
    """max / mean / median elementwise relative error and normwise error of x vs ref.

    Elementwise relative error uses max(|ref|, tiny) so exact zeros do not
    divide by zero; normwise = ||x - ref||_F / ||ref||_F."""
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    d = x - ref
    if ref_lo is not None:
        d = d - np.asarray(ref_lo, np.float64)
    a = np.abs(ref)
    tiny = np.finfo(np.float64).tiny
    rel = np.abs(d) / np.maximum(a, tiny)
    nrm = np.linalg.norm(ref)
    return {
        "max_rel": float(rel.max()) if rel.size else 0.0,
        "mean_rel": float(rel.mean()) if rel.size else 0.0,
        "median_rel": float(np.median(rel)) if rel.size else 0.0,
        "normwise": float(np.linalg.norm(d) / nrm) if nrm > 0 else float(np.linalg.norm(d)),
        "max_abs": float(np.abs(d).max()) if d.size else 0.0,
    }


# ------------------------------------------------------------------ reference


def ref_available():
    return os.path.exists(os.path.join(REF_DIR, "libref_cpu.so"))


_ref_cpu = None


def ref_cpu():
    """The reference's own Matrix<T> code (oracle/_ref/libref_cpu.so)."""
    global _ref_cpu
    if _ref_cpu is None:
        L = C.CDLL(os.path.join(REF_DIR, "libref_cpu.so"))
        dp, fp = C.POINTER(C.c_double), C.POINTER(C.c_float)
        L.ref_cpu_gemm_f64.argtypes = [C.c_int, C.c_int, C.c_int, dp, dp, dp]
        L.ref_cpu_gemm_f32.argtypes = [C.c_int, C.c_int, C.c_int, fp, fp, fp]
        L.ref_fill_random_f32.argtypes = [C.c_int, C.c_int, C.c_int, fp]
        L.ref_fill_random_f64.argtypes = [C.c_int, C.c_int, C.c_int, dp]
        _ref_cpu = L
    return _ref_cpu


def ref_product(A, B):
    """Matrix<double>::operator* of the reference on FP64 copies of A and B."""
    A, B = _f64(A), _f64(B)
    m, k = A.shape
    n = B.shape[1]
    out = np.empty((m, n), np.float64)
    ref_cpu().ref_cpu_gemm_f64(m, n, k, _p(A, C.c_double), _p(B, C.c_double), _p(out, C.c_double))
    return out


def ref_fill_random(seed, rows, cols, dtype=np.float32):
    out = np.empty((rows, cols), dtype)
    if dtype == np.float32:
        ref_cpu().ref_fill_random_f32(seed, rows, cols, _p(out, C.c_float))
    else:
        ref_cpu().ref_fill_random_f64(seed, rows, cols, _p(out, C.c_double))
    return out


class RefKernel:
    """One compile-time configuration of the reference kernel cosmaSgemm."""

    def __init__(self, tag):
        path = os.path.join(REF_DIR, "libref_gpu_%s.so" % tag)
        self.lib = C.CDLL(path)
        self.lib.ref_gpu_gemm.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int]
        self.lib.ref_gpu_gemm.restype = C.c_int
        cfg = (C.c_longlong * 11)()
        self.lib.ref_gpu_config(cfg)
        self.lib.ref_gpu_alpha.restype = C.c_double
        self.lib.ref_gpu_beta.restype = C.c_double
        keys = ["m", "n", "k", "tbm", "tbn", "tbk", "load_k", "split_k", "swizzle", "atomic", "elem"]
        self.config = dict(zip(keys, list(cfg)))
        self.alpha = self.lib.ref_gpu_alpha()
        self.beta = self.lib.ref_gpu_beta()

    def __call__(self, A_ptr, lda, B_ptr, ldb, C_ptr, ldc):
        return self.lib.ref_gpu_gemm(A_ptr, lda, B_ptr, ldb, C_ptr, ldc)


def ref_kernel_tags():
    if not os.path.isdir(REF_DIR):
        return []
    return sorted(f[len("libref_gpu_"):-3] for f in os.listdir(REF_DIR) if f.startswith("libref_gpu_") and f.endswith(".so"))
