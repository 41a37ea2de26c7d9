"""Failure detection without a GPU fault.  The test hook
CUCOSMA_FLAG_TEST_SKIP_STAGE makes the producer of every CTA leave its first
shared-memory stage unfilled, so the MMA issuer's wait on it (and, in turn,
the producer's and the epilogue's waits) run out after the short limit set
here.  The kernel must record CUCOSMA_STATUS_TIMEOUT in the device status
word, drain what it issued, release tensor memory and return; the context
must stay usable.  Host-side validation of the flag runs on the CPU."""
import numpy as np
import pytest

import cucosma_b200 as cc
import oracle
from tests._util import to_dev, uniform


def test_flag_rejected_on_native_path():
    d = cc.GemmDesc()
    cc.lib().cucosma_gemm_desc_init(d)
    d.m = d.n = d.k = 64
    d.lda = d.ldb = d.ldc = 64
    d.flags = cc.FLAG_TEST_SKIP_STAGE
    assert cc.lib().cucosma_gemm(d, None, None, None, None, 0, None) == cc.INVALID_VALUE
    d.flags = 1
    d.precision = 1
    assert cc.lib().cucosma_gemm(d, None, None, None, None, 0, None) == cc.INVALID_VALUE


@pytest.mark.gpu
@pytest.mark.parametrize("precision,dtype", [("bf16x3", np.float32), ("ozaki", np.float64)])
def test_skipped_stage_times_out_and_context_survives(cuda, precision, dtype):
    import torch

    m, n, k = 256, 384, 512
    A, B = uniform(50, (m, k), dtype), uniform(51, (k, n), dtype)
    dA, dB = to_dev(A), to_dev(B)
    cc.device_status()  # clear
    cc.set_wait_timeout_ns(20_000_000)  # 20 ms
    try:
        dC = to_dev(np.zeros((m, n), dtype))
        cc.gemm(dA, dB, dC, 1.0, 0.0, precision=precision, flags=cc.FLAG_TEST_SKIP_STAGE)
        torch.cuda.synchronize()  # the kernel returns: every wait is bounded
        s, code = cc.device_status()
        assert s == cc.TIMEOUT and code != 0, (s, hex(code))
    finally:
        cc.set_wait_timeout_ns(4_000_000_000)
    # the context is usable and the next call is correct and clean
    dC = to_dev(np.zeros((m, n), dtype))
    cc.gemm(dA, dB, dC, 1.0, 0.0, precision=precision)
    torch.cuda.synchronize()
    assert cc.device_status() == (cc.SUCCESS, 0)
    out = dC.cpu().numpy()
    ref = oracle.gemm(A, B, np.zeros((m, n), dtype), 1.0, 0.0)
    assert oracle.errors(out, ref)["normwise"] < (1e-4 if dtype == np.float32 else 1e-15)
