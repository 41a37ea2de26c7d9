"""ctypes bindings of the grouped-GEMM entry points (include/cucosma.h) and
a small Python mirror used by the tests and bench.py."""
from __future__ import annotations

import ctypes as C


class TuneResult(C.Structure):
    """Mirror of cucosma_tune_result."""

    _fields_ = [("split_k", C.c_int32), ("swizzle", C.c_int32), ("tile", C.c_int32), ("candidates", C.c_int32),
                ("occupancy", C.c_int32), ("reserved", C.c_int32), ("ms", C.c_double), ("tflops", C.c_double),
                ("l2_hit_rate", C.c_double), ("dram_bytes", C.c_double), ("counter_passes", C.c_int32),
                ("reserved2", C.c_int32)]

    def as_dict(self):
        return {f[0]: getattr(self, f[0]) for f in self._fields_ if not f[0].startswith("reserved")}


class Problem(C.Structure):
    """Mirror of cucosma_gemm_problem."""

    _fields_ = [("m", C.c_int64), ("n", C.c_int64), ("k", C.c_int64), ("lda", C.c_int64), ("ldb", C.c_int64),
                ("ldc", C.c_int64), ("A", C.c_void_p), ("B", C.c_void_p), ("C", C.c_void_p)]


def bind(L):
    from . import GemmDesc

    vp, sz = C.c_void_p, C.c_size_t
    P = C.POINTER(Problem)
    table = {
        "cucosma_grouped_workspace_size": ([C.POINTER(GemmDesc), P, C.c_int, C.POINTER(sz)], C.c_int),
        "cucosma_grouped_plan_create": ([C.POINTER(GemmDesc), P, C.c_int, vp, sz, C.POINTER(vp)], C.c_int),
        "cucosma_gemm_grouped": ([vp, vp], C.c_int),
        "cucosma_grouped_plan_destroy": ([vp], C.c_int),
        "cucosma_grouped_plan_get_tile": ([vp] + [C.POINTER(C.c_int32)] * 4, C.c_int),
        "cucosma_tune_grouped": ([C.POINTER(GemmDesc), P, C.c_int, vp, sz, C.POINTER(TuneResult), vp], C.c_int),
        "cucosma_tune": ([C.POINTER(GemmDesc), vp, vp, vp, vp, sz, C.c_int, C.POINTER(TuneResult), vp], C.c_int),
        "cucosma_tune_cache_save": ([C.c_char_p], C.c_int),
        "cucosma_tune_cache_load": ([C.c_char_p], C.c_int),
        "cucosma_tune_cache_clear": ([], C.c_int),
        "cucosma_tune_cache_size": ([], C.c_int),
        "cucosma_gemm_host_buffer_size": ([C.POINTER(GemmDesc), C.POINTER(sz)], C.c_int),
        "cucosma_gemm_host": ([C.POINTER(GemmDesc), vp, vp, vp, vp, sz, vp], C.c_int),
        "cucosma_gemm_backward_workspace_size": ([C.POINTER(GemmDesc), C.POINTER(sz)], C.c_int),
        "cucosma_gemm_backward": ([C.POINTER(GemmDesc), vp, vp, vp, C.c_int64, vp, C.c_int64, vp, C.c_int64, vp,
                                   C.c_int64, vp, sz, vp], C.c_int),
    }
    for name, (argtypes, restype) in table.items():
        f = getattr(L, name, None)
        if f is not None:
            f.argtypes = argtypes
            f.restype = restype


class GroupedPlan:
    """A grouped launch bound to device tensors: problems is a list of
    (A, B, C) row-major device tensors sharing dtype; the plan keeps them and
    its workspace alive.  __call__ enqueues the launch on the current stream."""

    def __init__(self, problems, precision="bf16x3", alpha=1.0, beta=0.0, epilogue="none", slices=0, tile=0):
        import torch

        from . import EPILOGUES, PRECISIONS, GemmDesc, _dtype_code, _ld, check, lib

        L = lib()
        self.problems = list(problems)
        arr = (Problem * len(self.problems))()
        for i, (A, B, Cm) in enumerate(self.problems):
            arr[i] = Problem(A.shape[0], B.shape[1], A.shape[1], _ld(A), _ld(B), _ld(Cm), A.data_ptr(), B.data_ptr(),
                             Cm.data_ptr())
        d = GemmDesc()
        L.cucosma_gemm_desc_init(C.byref(d))
        d.dtype = _dtype_code(self.problems[0][2])
        d.precision = PRECISIONS[precision]
        d.epilogue = EPILOGUES[epilogue]
        d.alpha, d.beta, d.slices, d.tile = float(alpha), float(beta), int(slices), int(tile)
        self.desc = d
        n = C.c_size_t(0)
        check(L.cucosma_grouped_workspace_size(C.byref(d), arr, len(self.problems), C.byref(n)),
              "cucosma_grouped_workspace_size")
        self.workspace = torch.empty(max(n.value, 256), dtype=torch.uint8, device=self.problems[0][2].device)
        h = C.c_void_p()
        check(L.cucosma_grouped_plan_create(C.byref(d), arr, len(self.problems), self.workspace.data_ptr(),
                                            self.workspace.numel(), C.byref(h)), "cucosma_grouped_plan_create")
        self.handle = h
        self._arr = arr
        self._lib = L

    def __call__(self, stream=None):
        from . import _stream_handle, check

        check(self._lib.cucosma_gemm_grouped(self.handle, _stream_handle(stream)), "cucosma_gemm_grouped")

    def tile(self):
        """(tile id, tile rows, tile columns, whether it came from the tuning cache)."""
        from . import check

        v = [C.c_int32() for _ in range(4)]
        check(self._lib.cucosma_grouped_plan_get_tile(self.handle, *[C.byref(x) for x in v]),
              "cucosma_grouped_plan_get_tile")
        return tuple(int(x.value) for x in v[:3]) + (bool(v[3].value),)

    def tune(self, stream=None):
        """cucosma_tune_grouped on this plan's problems (their C is
        overwritten) and workspace; returns the result as a dict."""
        from . import _stream_handle, check

        r = TuneResult()
        check(self._lib.cucosma_tune_grouped(C.byref(self.desc), self._arr, len(self.problems), self.workspace.data_ptr(),
                                             self.workspace.numel(), C.byref(r), _stream_handle(stream)),
              "cucosma_tune_grouped")
        return r.as_dict()

    def close(self):
        if getattr(self, "handle", None):
            self._lib.cucosma_grouped_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
