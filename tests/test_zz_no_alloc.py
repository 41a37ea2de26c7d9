"""GPU test of cucosma_sgemm_splitk_static, the entry point for callers that
must not allocate device memory (for example a plugin whose host framework
owns the whole device pool, or a latency-critical caller that cannot take
cudaMalloc's implicit synchronisation).  It keeps its split-K partial sums in
a fixed device array inside the library instead of a workspace.

Called through the C ABI twice in a row; each result is checked against the
regular entry point (cucosma_gemm with a caller-provided workspace and the
same split-K factor) within the error bound the native parity tests use.
This file is collected last on purpose, and passes on its own in a fresh
process as well as after the other tests."""
import ctypes as C

import numpy as np
import pytest

import cucosma_b200 as cc
from tests._util import bound, to_dev, uniform

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 16 << 20  # CUCOSMA_STATIC_SCRATCH_BYTES in include/cucosma.h


def _bind():
    L = cc.lib()
    f = L.cucosma_sgemm_splitk_static
    f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_float,
                  C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    f.restype = C.c_int
    return f


@pytest.mark.parametrize("shape,split_k", [((130, 129, 2000), 3), ((256, 256, 65536), 0), ((77, 61, 900), 7)])
def test_static_scratch_matches_regular_entry_point(cuda, shape, split_k):
    import torch

    f = _bind()
    m, n, k = shape
    A = uniform(41, (m, k))
    B = uniform(42, (k, n))
    Cin = uniform(43, (m, n))
    alpha, beta = 1.0, 0.5
    dA, dB = to_dev(A), to_dev(B)
    ref = to_dev(Cin)
    d = cc.make_desc(dA, dB, ref, alpha, beta, split_k=split_k)
    plan = cc.get_plan(d)
    assert plan["splits"] > 1, "the case must exercise the split-K scratch"
    cc.gemm(dA, dB, ref, alpha, beta, split_k=split_k)
    torch.cuda.synchronize()
    expect = ref.cpu().numpy()
    b = bound(A, B, Cin, alpha, beta, 0, np.float32, expect.astype(np.float64))
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        dC = to_dev(Cin)
        s = f(m, n, k, alpha, dA.data_ptr(), dA.stride(0), dB.data_ptr(), dB.stride(0), beta, dC.data_ptr(),
              dC.stride(0), split_k, stream)
        assert s == cc.SUCCESS, (call, s)
        torch.cuda.synchronize()
        out = dC.cpu().numpy()
        diff = np.abs(out.astype(np.float64) - expect)
        assert np.all(diff <= b), (call, float(diff.max()))
    st, code = cc.device_status()
    assert st == cc.SUCCESS, code


def test_static_scratch_rejects_oversized_problem(cuda):
    import torch

    f = _bind()
    m, n, k, split_k = 1024, 1024, 8192, 8  # 8 * 1024 * 1024 * 4 B = 32 MiB of partials
    assert split_k * m * n * 4 > SCRATCH_BYTES
    dA = torch.zeros((m, k), device="cuda")
    dB = torch.zeros((k, n), device="cuda")
    dC = torch.full((m, n), 7.0, device="cuda")
    s = f(m, n, k, 1.0, dA.data_ptr(), k, dB.data_ptr(), n, 0.0, dC.data_ptr(), n, split_k, None)
    assert s == cc.WORKSPACE_TOO_SMALL
    torch.cuda.synchronize()
    assert bool((dC == 7.0).all())  # nothing was launched
