"""CPU tests of the C ABI boundary: the library loads, exports every entry
point include/*.h declares, and rejects bad arguments before touching a GPU
(validation runs first, so these calls never reach CUDA)."""
import ctypes as C
import glob
import os
import re

import pytest

import cucosma_b200 as cc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        names.update(re.findall(r"CUCOSMA_API\s+[\w\s\*]+?\b(cucosma_\w+)\s*\(", txt))
    return sorted(names)


def test_library_loads_and_exports_every_declared_symbol():
    L = cc.lib()
    names = declared_symbols()
    assert "cucosma_gemm" in names and "cucosma_sgemm" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_version_and_error_strings():
    L = cc.lib()
    assert L.cucosma_get_version() >= 100
    for s in range(10):
        assert len(L.cucosma_get_error_string(s)) > 0


def _desc(**kw):
    d = cc.GemmDesc()
    cc.lib().cucosma_gemm_desc_init(C.byref(d))
    d.m, d.n, d.k, d.lda, d.ldb, d.ldc = 64, 64, 64, 64, 64, 64
    for a, b in kw.items():
        setattr(d, a, b)
    return d


FAKE = 0x10000  # aligned, never dereferenced: validation returns first


def _gemm(d, A=FAKE, B=FAKE, Cp=FAKE):
    return cc.lib().cucosma_gemm(C.byref(d) if d is not None else None, A, B, Cp, None, 0, None)


def test_defaults():
    d = _desc()
    assert d.alpha == 1.0 and d.beta == 0.0 and d.dtype == cc.R_32F and d.precision == 0


@pytest.mark.parametrize(
    "kw,status",
    [
        (dict(m=-1), cc.INVALID_VALUE),
        (dict(k=-5), cc.INVALID_VALUE),
        (dict(lda=10), cc.INVALID_VALUE),
        (dict(ldb=10), cc.INVALID_VALUE),
        (dict(ldc=10), cc.INVALID_VALUE),
        (dict(dtype=7), cc.INVALID_VALUE),
        (dict(precision=9), cc.INVALID_VALUE),
        (dict(epilogue=5), cc.INVALID_VALUE),
        (dict(flags=1), cc.INVALID_VALUE),
        (dict(slices=2), cc.INVALID_VALUE),
        (dict(split_k=-1), cc.INVALID_VALUE),
        (dict(lda=65), cc.MISALIGNED),
        (dict(ldc=66), cc.MISALIGNED),
        (dict(dtype=cc.R_64F, precision=cc.PRECISIONS["bf16x3"]), cc.NOT_SUPPORTED),
        (dict(dtype=cc.R_32F, precision=cc.PRECISIONS["ozaki"]), cc.NOT_SUPPORTED),
    ],
)
def test_validation_rejects_before_launch(kw, status):
    assert _gemm(_desc(**kw)) == status


def test_null_arguments():
    assert _gemm(None) == cc.INVALID_VALUE
    assert _gemm(_desc(), A=None) == cc.INVALID_VALUE
    assert _gemm(_desc(), Cp=None) == cc.INVALID_VALUE
    assert _gemm(_desc(), A=FAKE + 4) == cc.MISALIGNED


def test_empty_problem_is_a_no_op():
    # m == 0 or n == 0: nothing to do, nothing launched.
    assert _gemm(_desc(m=0), A=None, B=None, Cp=None) == cc.SUCCESS
    assert _gemm(_desc(n=0), A=None, B=None, Cp=None) == cc.SUCCESS


def test_workspace_size_rejects_bad_desc():
    n = C.c_size_t(0)
    assert cc.lib().cucosma_gemm_workspace_size(None, C.byref(n)) == cc.INVALID_VALUE
    assert cc.lib().cucosma_gemm_workspace_size(C.byref(_desc(m=-3)), C.byref(n)) == cc.INVALID_VALUE


def test_timeout_setter_validates():
    assert cc.lib().cucosma_set_wait_timeout_ns(0) == cc.INVALID_VALUE
