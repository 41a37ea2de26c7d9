"""cucosma_b200 -- cuCOSMA-compatible GEMM for NVIDIA B200 (sm_100a).

The product is the native library ``cucosma_b200/libcucosma.so`` (CUDA
kernels + the C ABI of ``include/cucosma.h``).  This module is a thin ctypes
binding used by Python callers, the tests and bench.py: it passes device
pointers, strides and the caller's CUDA stream, and raises ``CucosmaError``
on any non-success status.  There is no fallback: if the library is missing
or fails to load, importing the binding raises.

Reference interface mirrored: ``cosmaSgemm(A, lda, B, ldb, C, ldc)``
(Kernel/cuda/src/cuCOSMAV100.cuh:2774) with M, N, K, ALPHA, BETA taken from
the tensors and arguments instead of config.h macros.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcucosma.so")

SUCCESS, INVALID_VALUE, MISALIGNED, NOT_SUPPORTED, WORKSPACE_TOO_SMALL = 0, 1, 2, 3, 4
LAUNCH_FAILED, TIMEOUT, ARCH_MISMATCH, ALLOC_FAILED, INTERNAL_ERROR = 5, 6, 7, 8, 9

R_32F, R_64F = 0, 1
PRECISIONS = {"native": 0, "bf16x3": 1, "bf16x6": 2, "ozaki": 3}
EPILOGUES = {"none": 0, "sigmoid": 1, "relu": 2}


class CucosmaError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        msg = lib().cucosma_get_error_string(status).decode()
        super().__init__("%s: status %d (%s)" % (what or "cucosma", status, msg))


class GemmDesc(C.Structure):
    """Mirror of cucosma_gemm_desc (include/cucosma.h)."""

    _fields_ = [
        ("m", C.c_int64), ("n", C.c_int64), ("k", C.c_int64),
        ("lda", C.c_int64), ("ldb", C.c_int64), ("ldc", C.c_int64),
        ("dtype", C.c_int32), ("precision", C.c_int32), ("slices", C.c_int32), ("epilogue", C.c_int32),
        ("alpha", C.c_double), ("beta", C.c_double),
        ("split_k", C.c_int32), ("swizzle", C.c_int32), ("tile", C.c_int32), ("flags", C.c_int32),
    ]


class PlanInfo(C.Structure):
    """Mirror of cucosma_plan_info (include/cucosma.h)."""

    _fields_ = [
        ("path", C.c_int32), ("tile_m", C.c_int32), ("tile_n", C.c_int32), ("tile_k", C.c_int32),
        ("splits", C.c_int32), ("band", C.c_int32), ("slices", C.c_int32), ("launches", C.c_int32),
        ("kchunk", C.c_int64), ("kpad", C.c_int64),
        ("workspace_bytes", C.c_uint64), ("off_a", C.c_uint64), ("off_b", C.c_uint64), ("off_ea", C.c_uint64),
        ("off_eb", C.c_uint64), ("off_part", C.c_uint64), ("off_choice", C.c_uint64),
        ("layout_slices", C.c_int32), ("fused", C.c_int32),
    ]

    def as_dict(self):
        return {f[0]: getattr(self, f[0]) for f in self._fields_}


_lib = None

# Every symbol include/cucosma.h declares; checked when the library loads.
EXPORTS = [
    "cucosma_gemm_desc_init", "cucosma_gemm_workspace_size", "cucosma_gemm", "cucosma_sgemm", "cucosma_dgemm",
    "cucosma_device_status", "cucosma_set_wait_timeout_ns", "cucosma_get_error_string", "cucosma_get_version",
    "cucosma_launch_count", "cucosma_profile_start", "cucosma_profile_stop", "cucosma_gemm_get_plan",
    "cucosma_gemm_managed",
]


def lib():
    """Load libcucosma.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("cucosma_b200: %s not built (run __graft_entry__.build())" % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    vp, sz = C.c_void_p, C.c_size_t
    L.cucosma_gemm_desc_init.argtypes = [C.POINTER(GemmDesc)]
    L.cucosma_gemm_desc_init.restype = None
    L.cucosma_gemm_workspace_size.argtypes = [C.POINTER(GemmDesc), C.POINTER(sz)]
    L.cucosma_gemm.argtypes = [C.POINTER(GemmDesc), vp, vp, vp, vp, sz, vp]
    L.cucosma_sgemm.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, vp, C.c_int, vp, C.c_int, C.c_float, vp, C.c_int, vp]
    L.cucosma_dgemm.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, vp, C.c_int, vp, C.c_int, C.c_double, vp, C.c_int, vp]
    L.cucosma_device_status.argtypes = [C.POINTER(C.c_int)]
    L.cucosma_set_wait_timeout_ns.argtypes = [C.c_uint64]
    L.cucosma_get_error_string.argtypes = [C.c_int]
    L.cucosma_get_error_string.restype = C.c_char_p
    L.cucosma_get_version.restype = C.c_int
    L.cucosma_launch_count.restype = C.c_ulonglong
    L.cucosma_profile_stop.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_int64)]
    L.cucosma_gemm_get_plan.argtypes = [C.POINTER(GemmDesc), C.POINTER(PlanInfo)]
    L.cucosma_gemm_managed.argtypes = [C.POINTER(GemmDesc), vp, vp, vp, vp]
    for name in EXPORTS:
        if name not in ("cucosma_gemm_desc_init", "cucosma_get_error_string", "cucosma_get_version",
                        "cucosma_launch_count"):
            getattr(L, name).restype = C.c_int
    _lib = L
    _bind_optional(L)
    return L


def _bind_optional(L):
    """Entry points added by later modules (grouped, sigmoid fwd/bwd, tuner)."""
    from . import _ext

    _ext.bind(L)


def check(status, what=""):
    if status != SUCCESS:
        raise CucosmaError(status, what)


def _stream_handle(stream):
    if stream is None:
        import torch

        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


def _dtype_code(t):
    import torch

    if t.dtype == torch.float32:
        return R_32F
    if t.dtype == torch.float64:
        return R_64F
    raise TypeError("cucosma: only float32 / float64 matrices (got %s)" % t.dtype)


def _ld(t):
    if t.dim() != 2 or t.stride(1) != 1:
        raise ValueError("cucosma: matrices must be 2-D row-major with unit column stride")
    return t.stride(0) if t.shape[0] > 1 else max(t.stride(0), t.shape[1])


FLAG_TEST_SKIP_STAGE = 1 << 30  # CUCOSMA_FLAG_TEST_SKIP_STAGE: failure-path test hook


def make_desc(A, B, Cm, alpha=1.0, beta=0.0, precision="native", epilogue="none", split_k=0, swizzle=0,
              slices=0, tile=0, flags=0):
    m, k = A.shape
    k2, n = B.shape
    if k != k2 or tuple(Cm.shape) != (m, n):
        raise ValueError("cucosma: shape mismatch A%s B%s C%s" % (tuple(A.shape), tuple(B.shape), tuple(Cm.shape)))
    d = GemmDesc()
    lib().cucosma_gemm_desc_init(C.byref(d))
    d.m, d.n, d.k = m, n, k
    d.lda, d.ldb, d.ldc = _ld(A), _ld(B), _ld(Cm)
    d.dtype = _dtype_code(Cm)
    d.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    d.epilogue = EPILOGUES[epilogue] if isinstance(epilogue, str) else int(epilogue)
    d.alpha, d.beta = float(alpha), float(beta)
    d.split_k, d.swizzle, d.slices, d.tile, d.flags = int(split_k), int(swizzle), int(slices), int(tile), int(flags)
    return d


def get_plan(desc):
    info = PlanInfo()
    check(lib().cucosma_gemm_get_plan(C.byref(desc), C.byref(info)), "cucosma_gemm_get_plan")
    return info.as_dict()


def workspace_size(desc):
    n = C.c_size_t(0)
    check(lib().cucosma_gemm_workspace_size(C.byref(desc), C.byref(n)), "cucosma_gemm_workspace_size")
    return n.value


def alloc_workspace(desc, device=None):
    import torch

    n = workspace_size(desc)
    if n == 0:
        return None
    return torch.empty(n, dtype=torch.uint8, device=device or "cuda")


def gemm(A, B, Cm, alpha=1.0, beta=0.0, precision="native", epilogue="none", split_k=0, swizzle=0, slices=0,
         tile=0, workspace=None, stream=None, flags=0):
    """C <- epi(alpha*A@B + beta*C) in place on device tensors; returns C."""
    d = make_desc(A, B, Cm, alpha, beta, precision, epilogue, split_k, swizzle, slices, tile, flags)
    if workspace is None:
        workspace = alloc_workspace(d, Cm.device)
    ws_ptr = workspace.data_ptr() if workspace is not None else None
    ws_n = workspace.numel() * workspace.element_size() if workspace is not None else 0
    check(lib().cucosma_gemm(C.byref(d), A.data_ptr(), B.data_ptr(), Cm.data_ptr(), ws_ptr, ws_n,
                             _stream_handle(stream)), "cucosma_gemm")
    return Cm


def host_desc(A, B, Cm, alpha=1.0, beta=0.0, precision="native", epilogue="none", split_k=0, slices=0, tile=0):
    """Descriptor for cucosma_gemm_host from host (CPU) tensors: ld* are their row strides."""
    return make_desc(A, B, Cm, alpha, beta, precision, epilogue, split_k, 0, slices, tile)


def host_buffer(desc, device=None):
    """Device buffer of cucosma_gemm_host_buffer_size bytes (256-byte aligned)."""
    import torch

    n = C.c_size_t(0)
    check(lib().cucosma_gemm_host_buffer_size(C.byref(desc), C.byref(n)), "cucosma_gemm_host_buffer_size")
    return torch.empty(n.value, dtype=torch.uint8, device=device or "cuda")


def gemm_host(A, B, Cm, alpha=1.0, beta=0.0, precision="native", epilogue="none", split_k=0, slices=0, tile=0,
              buffer=None, stream=None):
    """C <- epi(alpha*A@B + beta*C) on host (CPU, ideally pinned) tensors through
    cucosma_gemm_host: the copies in and out overlap the row-block GEMMs.
    Asynchronous on the stream; synchronise before reading C."""
    d = host_desc(A, B, Cm, alpha, beta, precision, epilogue, split_k, slices, tile)
    if buffer is None:
        buffer = host_buffer(d)
    check(lib().cucosma_gemm_host(C.byref(d), A.data_ptr(), B.data_ptr(), Cm.data_ptr(), buffer.data_ptr(),
                                  buffer.numel(), _stream_handle(stream)), "cucosma_gemm_host")
    return Cm


def cosma_sgemm(A, B, Cm, alpha=1.0, beta=0.0, stream=None):
    """The reference-shaped entry point: cosmaSgemm(A, lda, B, ldb, C, ldc) with
    M, N, K from the tensor shapes (FP32 -> cucosma_sgemm, FP64 -> cucosma_dgemm)."""
    m, k = A.shape
    n = B.shape[1]
    f = lib().cucosma_sgemm if Cm.dtype.itemsize == 4 else lib().cucosma_dgemm
    check(f(m, n, k, alpha, A.data_ptr(), _ld(A), B.data_ptr(), _ld(B), beta, Cm.data_ptr(), _ld(Cm),
            _stream_handle(stream)), "cosmaSgemm")
    return Cm


def device_status():
    code = C.c_int(0)
    s = lib().cucosma_device_status(C.byref(code))
    return s, code.value


def launch_count():
    """Kernels the library has enqueued in this process."""
    return int(lib().cucosma_launch_count())


def profile_start():
    check(lib().cucosma_profile_start(), "cucosma_profile_start")


def profile_stop():
    """(summed main-kernel milliseconds, timed launches) since profile_start()."""
    ms, n = C.c_double(0), C.c_int64(0)
    check(lib().cucosma_profile_stop(C.byref(ms), C.byref(n)), "cucosma_profile_stop")
    return ms.value, n.value


def tune(A, B, Cm, alpha=1.0, beta=0.0, precision="native", slices=0, max_candidates=0, workspace=None,
         stream=None):
    """Measure candidate configurations of this GEMM on the device and cache
    the fastest (C is overwritten).  Returns the cucosma_tune_result fields."""
    import torch

    from ._ext import TuneResult

    d = make_desc(A, B, Cm, alpha, beta, precision=precision, slices=slices)
    if workspace is None:
        # room for the largest split-K candidate
        biggest = 0
        for sk in (1, 2, 4, 8, 16, 32, 64):
            dd = make_desc(A, B, Cm, alpha, beta, precision=precision, slices=slices, split_k=sk)
            biggest = max(biggest, workspace_size(dd))
        workspace = torch.empty(max(biggest, 256), dtype=torch.uint8, device=Cm.device)
    r = TuneResult()
    check(lib().cucosma_tune(C.byref(d), A.data_ptr(), B.data_ptr(), Cm.data_ptr(), workspace.data_ptr(),
                             workspace.numel(), int(max_candidates), C.byref(r), _stream_handle(stream)),
          "cucosma_tune")
    return r.as_dict()


def tune_cache_save(path):
    check(lib().cucosma_tune_cache_save(os.fsencode(path)), "cucosma_tune_cache_save")


def tune_cache_load(path):
    check(lib().cucosma_tune_cache_load(os.fsencode(path)), "cucosma_tune_cache_load")


def tune_cache_clear():
    check(lib().cucosma_tune_cache_clear(), "cucosma_tune_cache_clear")


def tune_cache_size():
    return int(lib().cucosma_tune_cache_size())


def gemm_backward(A, B, Y, dY, dA=None, dB=None, alpha=1.0, precision="bf16x3", epilogue="sigmoid", workspace=None,
                  stream=None):
    """Gradients of Y = epi(alpha*A@B + beta*C0): dA = G@B^T, dB = A^T@G with
    G = alpha * dY * epi'(Z) (epi' from the saved Y).  Writes dA / dB in place."""
    import torch

    L = lib()
    d = make_desc(A, B, Y, alpha, 0.0, precision=precision, epilogue=epilogue)
    if workspace is None:
        n = C.c_size_t(0)
        check(L.cucosma_gemm_backward_workspace_size(C.byref(d), C.byref(n)), "cucosma_gemm_backward_workspace_size")
        workspace = torch.empty(max(n.value, 256), dtype=torch.uint8, device=Y.device)
    ws_n = workspace.numel() * workspace.element_size()
    check(L.cucosma_gemm_backward(C.byref(d), A.data_ptr(), B.data_ptr(), Y.data_ptr(), _ld(Y), dY.data_ptr(), _ld(dY),
                                  dA.data_ptr() if dA is not None else None, _ld(dA) if dA is not None else 0,
                                  dB.data_ptr() if dB is not None else None, _ld(dB) if dB is not None else 0,
                                  workspace.data_ptr(), ws_n, _stream_handle(stream)), "cucosma_gemm_backward")
    return dA, dB


def grouped(problems, precision="bf16x3", alpha=1.0, beta=0.0, epilogue="none", slices=0, tile=0):
    """Plan a grouped launch over [(A, B, C), ...] device tensors; call the
    returned object to enqueue it (two or three kernels, graph-capturable).
    tile 0 takes the tuner's choice for this batch when it has one."""
    from ._ext import GroupedPlan

    return GroupedPlan(problems, precision, alpha, beta, epilogue, slices, tile)


def set_wait_timeout_ns(ns):
    check(lib().cucosma_set_wait_timeout_ns(int(ns)), "cucosma_set_wait_timeout_ns")
