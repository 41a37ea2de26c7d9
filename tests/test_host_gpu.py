"""cucosma_gemm_host: operands and result in host memory, copies overlapped
with row-block GEMMs.  Checked against the oracle's bound for every path,
with beta != 0 (C copied in), ragged row blocks, padded host rows, pinned
and pageable memory, and two calls sharing one device buffer."""
import numpy as np
import pytest

import cucosma_b200 as cc
import oracle
from tests._util import bf16_bound, check_against_oracle, uniform

pytestmark = pytest.mark.gpu


def host(x, pinned=True, pad=0):
    import torch

    t = torch.zeros((x.shape[0], x.shape[1] + pad), dtype=getattr(torch, str(x.dtype)))
    if pinned:
        t = t.pin_memory()
    v = t[:, :x.shape[1]]
    v.copy_(torch.from_numpy(np.ascontiguousarray(x)))
    return v


CASES = [("native", np.float32, 1000, 300, 500), ("native", np.float64, 777, 129, 260),
         ("native", np.float32, 3000, 64, 40), ("bf16x3", np.float32, 1500, 700, 900),
         ("bf16x6", np.float32, 2100, 300, 700), ("ozaki", np.float64, 900, 256, 320),
         ("ozaki-adaptive", np.float64, 1300, 200, 300)]


@pytest.mark.parametrize("case", CASES, ids=["%s_%s_%dx%dx%d" % (c[0], np.dtype(c[1]).name, *c[2:]) for c in CASES])
@pytest.mark.parametrize("pinned", [True, False], ids=["pinned", "pageable"])
def test_gemm_host(cuda, case, pinned):
    import torch

    prec, dtype, m, n, k = case
    A, B, Cin = uniform(1, (m, k), dtype), uniform(2, (k, n), dtype), uniform(3, (m, n), dtype)
    hA, hB = host(A, pinned, pad=4), host(B, pinned)
    hC = host(Cin, pinned, pad=2)
    # row blocks after the first reuse B's planes / slices prepared by the first
    cc.gemm_host(hA, hB, hC, 1.25, 0.5, precision=prec.split("-")[0], slices=8 if prec == "ozaki" else 0)
    torch.cuda.synchronize()
    out = hC.numpy()
    if prec == "native":
        check_against_oracle(out, A, B, Cin, 1.25, 0.5, oracle.EPI_NONE, dtype)
    elif prec in ("bf16x3", "bf16x6"):
        ref, b = bf16_bound(A, B, Cin, 1.25, 0.5, 2 if prec == "bf16x3" else 3)
        assert np.all(np.abs(out - ref) <= b)
    else:
        ref = oracle.gemm(A, B, Cin, 1.25, 0.5)
        assert oracle.errors(out, ref)["normwise"] < 1e-15
    assert cc.device_status() == (cc.SUCCESS, 0)


def test_gemm_host_two_calls_share_a_buffer(cuda):
    import torch

    m, n, k = 2048, 512, 1024
    A1, A2, B = uniform(4, (m, k)), uniform(5, (m, k)), uniform(6, (k, n))
    hA1, hA2, hB = host(A1), host(A2), host(B)
    hC1, hC2 = host(np.zeros((m, n), np.float32)), host(np.zeros((m, n), np.float32))
    d = cc.host_desc(hA1, hB, hC1)
    buf = cc.host_buffer(d)
    cc.gemm_host(hA1, hB, hC1, buffer=buf)
    cc.gemm_host(hA2, hB, hC2, buffer=buf)  # ordered after the first on the same stream
    torch.cuda.synchronize()
    Z = np.zeros((m, n), np.float32)
    check_against_oracle(hC1.numpy(), A1, B, Z, 1.0, 0.0, oracle.EPI_NONE, np.float32)
    check_against_oracle(hC2.numpy(), A2, B, Z, 1.0, 0.0, oracle.EPI_NONE, np.float32)


def test_gemm_host_rejects_small_buffer(cuda):
    import torch

    A, B = uniform(7, (300, 100)), uniform(8, (100, 200))
    hA, hB, hC = host(A), host(B), host(np.zeros((300, 200), np.float32))
    d = cc.host_desc(hA, hB, hC)
    small = torch.empty(1024, dtype=torch.uint8, device="cuda")
    s = cc.lib().cucosma_gemm_host(d, hA.data_ptr(), hB.data_ptr(), hC.data_ptr(), small.data_ptr(), 1024, None)
    assert s == cc.WORKSPACE_TOO_SMALL


@pytest.mark.parametrize("precision", ["native", "bf16x6"])
def test_gemm_host_two_threads(cuda, precision):
    """Two host threads call cucosma_gemm_host at the same time, each with its
    own operands, device buffer and stream, three times each: every call
    orders its copies and GEMMs with events of its own, so both results stay
    correct."""
    import threading

    import torch

    m, n, k = 1536, 384, 512
    jobs = []
    for t in range(2):
        A, B = uniform(10 + t, (m, k)), uniform(20 + t, (k, n))
        hA, hB, hC = host(A), host(B), host(np.zeros((m, n), np.float32))
        buf = cc.host_buffer(cc.host_desc(hA, hB, hC, precision=precision))
        jobs.append((A, B, hA, hB, hC, buf, torch.cuda.Stream()))
    errors = []

    def work(j):
        A, B, hA, hB, hC, buf, st = jobs[j]
        try:
            for _ in range(3):
                cc.gemm_host(hA, hB, hC, precision=precision, buffer=buf, stream=st)
            st.synchronize()
        except Exception as ex:  # reported below, on the test's thread
            errors.append(ex)

    threads = [threading.Thread(target=work, args=(j,)) for j in range(2)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    assert not errors, errors
    torch.cuda.synchronize()
    Z = np.zeros((m, n), np.float32)
    for A, B, _, _, hC, _, _ in jobs:
        if precision == "native":
            check_against_oracle(hC.numpy(), A, B, Z, 1.0, 0.0, oracle.EPI_NONE, np.float32)
        else:
            ref, b = bf16_bound(A, B, Z, 1.0, 0.0, 3)
            assert np.all(np.abs(hC.numpy() - ref) <= b)
    assert cc.device_status() == (cc.SUCCESS, 0)
