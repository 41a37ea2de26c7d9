"""GPU tests of the forward/backward pair through the C ABI.

Forward: Y = sigmoid(alpha * A@B) (cucosma_gemm, fused epilogue).  Backward:
dA = G@B^T, dB = A^T@G with G = alpha * dY * Y(1-Y) fused into the operand
pre-pass (cucosma_gemm_backward).  Checked against FP64 finite differences of
L = sum(dY * Y) at M = N = K = 64 and 256, against the analytic FP64
gradients for the ReLU / identity epilogues, and against the reference kernel
cosmaSgemm applied to explicitly transposed operands (oracle/_ref)."""
import numpy as np
import pytest

import cucosma_b200 as cc
import oracle
from tests._util import to_dev, uniform

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def short_waits(cuda):
    cc.set_wait_timeout_ns(2_000_000_000)
    yield
    s, code = cc.device_status()
    assert s == cc.SUCCESS, "device status %d code 0x%x" % (s, code)


def sig(x):
    return 1.0 / (1.0 + np.exp(-x))


def fwd_bwd(A, B, W, alpha, precision, epilogue):
    import torch

    m, k = A.shape
    n = B.shape[1]
    dA_, dB_, dY = to_dev(A), to_dev(B), to_dev(W)
    Y = to_dev(np.zeros((m, n), np.float32))
    cc.gemm(dA_, dB_, Y, alpha, 0.0, precision=precision, epilogue=epilogue)
    gA = to_dev(np.zeros((m, k), np.float32))
    gB = to_dev(np.zeros((k, n), np.float32))
    cc.gemm_backward(dA_, dB_, Y, dY, gA, gB, alpha=alpha, precision=precision, epilogue=epilogue)
    torch.cuda.synchronize()
    return Y.cpu().numpy(), gA.cpu().numpy(), gB.cpu().numpy()


@pytest.mark.parametrize("n", [64, 256])
@pytest.mark.parametrize("precision,rtol", [("bf16x3", 2e-4), ("bf16x6", 2e-5)])
def test_finite_differences(n, precision, rtol):
    alpha = 1.5
    A = uniform(1, (n, n), lo=-0.1, hi=0.1)
    B = uniform(2, (n, n), lo=-0.1, hi=0.1)
    W = uniform(3, (n, n))
    Y, gA, gB = fwd_bwd(A, B, W, alpha, precision, "sigmoid")
    A64, B64, W64 = A.astype(np.float64), B.astype(np.float64), W.astype(np.float64)
    Z = alpha * oracle.gemm(A64, B64)
    assert np.abs(Y - sig(Z)).max() < 1e-5
    G = alpha * W64 * sig(Z) * (1 - sig(Z))
    dA64, dB64 = oracle.gemm(G, B64.T), oracle.gemm(A64.T, G)
    # central differences of L = sum(W * sigmoid(Z)) in FP64 on sampled entries;
    # perturbing A[i, j] changes row i of Z only, B[j, c] column c only.
    h = 1e-6
    rng = np.random.default_rng(4)
    for _ in range(48):
        i, j = rng.integers(0, n, 2)
        d = (np.sum(W64[i] * sig(Z[i] + alpha * h * B64[j])) - np.sum(W64[i] * sig(Z[i] - alpha * h * B64[j]))) / (2 * h)
        assert abs(d - dA64[i, j]) <= 1e-8 * (1 + abs(d))
        assert abs(gA[i, j] - d) <= rtol * np.abs(dA64).max()
        d = (np.sum(W64[:, j] * sig(Z[:, j] + alpha * h * A64[:, i])) -
             np.sum(W64[:, j] * sig(Z[:, j] - alpha * h * A64[:, i]))) / (2 * h)
        assert abs(d - dB64[i, j]) <= 1e-8 * (1 + abs(d))
        assert abs(gB[i, j] - d) <= rtol * np.abs(dB64).max()
    # every entry against the analytic FP64 gradient
    assert np.abs(gA - dA64).max() <= rtol * np.abs(dA64).max()
    assert np.abs(gB - dB64).max() <= rtol * np.abs(dB64).max()


@pytest.mark.parametrize("epilogue", ["relu", "none"])
def test_other_epilogues(epilogue):
    m, n, k = 130, 70, 90
    alpha = 0.75
    A = uniform(5, (m, k))
    B = uniform(6, (k, n))
    W = uniform(7, (m, n))
    Y, gA, gB = fwd_bwd(A, B, W, alpha, "bf16x6", epilogue)
    Z = alpha * oracle.gemm(A, B)
    d = (Z > 0).astype(np.float64) if epilogue == "relu" else np.ones_like(Z)
    if epilogue == "relu":
        d = (Y > 0).astype(np.float64)  # the mask the backward reads
    G = alpha * W.astype(np.float64) * d
    dA64, dB64 = oracle.gemm(G, B.T), oracle.gemm(A.T, G)
    assert np.abs(gA - dA64).max() <= 2e-5 * np.abs(dA64).max()
    assert np.abs(gB - dB64).max() <= 2e-5 * np.abs(dB64).max()


def test_only_one_gradient():
    import torch

    A = uniform(8, (64, 48))
    B = uniform(9, (48, 40))
    W = uniform(10, (64, 40))
    dA_, dB_, dY = to_dev(A), to_dev(B), to_dev(W)
    Y = to_dev(np.zeros((64, 40), np.float32))
    cc.gemm(dA_, dB_, Y, 1.0, 0.0, precision="bf16x3", epilogue="sigmoid")
    gB = to_dev(np.zeros((48, 40), np.float32))
    cc.gemm_backward(dA_, dB_, Y, dY, None, gB, precision="bf16x3", epilogue="sigmoid")
    torch.cuda.synchronize()
    Yh = Y.cpu().numpy().astype(np.float64)
    G = W * Yh * (1 - Yh)
    ref = oracle.gemm(A.T, G)
    assert np.abs(gB.cpu().numpy() - ref).max() <= 2e-4 * np.abs(ref).max()


@pytest.mark.skipif("f32_1024_a1b0" not in oracle.ref_kernel_tags(), reason="oracle/_ref not built")
def test_against_reference_kernel_on_transposed_operands():
    """dA = G @ B^T and dB = A^T @ G also through the reference kernel
    (1024^3, alpha 1, beta 0), fed with G computed on the host from the saved
    forward output and explicitly transposed operands."""
    import torch

    n = 1024
    A = uniform(11, (n, n), lo=-0.1, hi=0.1)
    B = uniform(12, (n, n), lo=-0.1, hi=0.1)
    W = uniform(13, (n, n))
    Y, gA, gB = fwd_bwd(A, B, W, 1.0, "bf16x3", "sigmoid")
    G = (np.float32(1.0) * W) * (Y * (np.float32(1.0) - Y))  # the pre-pass's FP32 formula
    ref = oracle.RefKernel("f32_1024_a1b0")

    def ref_gemm(X, Z):
        dX, dZ = to_dev(np.ascontiguousarray(X), ld=n), to_dev(np.ascontiguousarray(Z), ld=n)
        dC = to_dev(np.zeros((n, n), np.float32), ld=n)
        assert ref(dX.data_ptr(), n, dZ.data_ptr(), n, dC.data_ptr(), n) == 0
        torch.cuda.synchronize()
        return dC.cpu().numpy()

    u = 2.0 ** -24
    for ours, X, Z in ((gA, G, B.T), (gB, A.T, G)):
        exact = oracle.gemm(X, Z)
        absxz = oracle.gemm(np.abs(X), np.abs(Z))
        r = ref_gemm(X, Z)
        assert np.all(np.abs(r - exact) <= (n + 2) * u * absxz + 1e-30)  # reference: FP32 SIMT bound
        assert np.all(np.abs(ours - exact) <= (3.1 * 2.0 ** -16 + 6 * (n + 2) * u) * absxz + 1e-30)
        print("max |ours - reference| / max|ref|:", np.abs(ours - r).max() / np.abs(r).max())


def test_backward_rejects_bad_arguments():
    import ctypes as C

    L = cc.lib()
    d = cc.GemmDesc()
    L.cucosma_gemm_desc_init(C.byref(d))
    d.m = d.n = d.k = d.lda = d.ldb = d.ldc = 64
    d.precision = cc.PRECISIONS["native"]
    n = C.c_size_t(0)
    assert L.cucosma_gemm_backward_workspace_size(C.byref(d), C.byref(n)) == cc.NOT_SUPPORTED
    d.precision = cc.PRECISIONS["bf16x3"]
    assert L.cucosma_gemm_backward_workspace_size(C.byref(d), C.byref(n)) == cc.SUCCESS
    f = 0x10000
    st = L.cucosma_gemm_backward(C.byref(d), f, f, f, 64, f, 64, f + 4, 64, None, 0, f, n.value, None)
    assert st == cc.MISALIGNED
    st = L.cucosma_gemm_backward(C.byref(d), f, f, f, 64, None, 64, f, 64, None, 0, f, n.value, None)
    assert st == cc.INVALID_VALUE


def test_backward_with_tuned_subproblem_fits_queried_workspace(tmp_path):
    """A tuning-cache entry for the dB product (k x n x m, BF16x3) that forces
    one split: the queried workspace then has no split-K partials region, and
    the backward call must run the product with that same tuned plan.  A
    guard band after the queried workspace must stay untouched and the
    gradients must still match FP64."""
    import ctypes as C

    import torch

    m, n, k = 4096, 512, 512
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    cache = tmp_path / "tune.txt"
    # v1 <sms> <dtype> <precision> <slices> <m> <n> <k> <split_k> <swizzle> <tile> <ms>: the dB product
    cache.write_text("v1 %d 0 1 0 %d %d %d 1 0 0 1.0\n" % (sms, k, n, m))
    cc.tune_cache_clear()
    try:
        cc.tune_cache_load(str(cache))
        A = uniform(14, (m, k), lo=-0.1, hi=0.1)
        B = uniform(15, (k, n), lo=-0.1, hi=0.1)
        W = uniform(16, (m, n))
        dA_, dB_, dY = to_dev(A), to_dev(B), to_dev(W)
        Y = to_dev(np.zeros((m, n), np.float32))
        cc.gemm(dA_, dB_, Y, 1.0, 0.0, precision="bf16x3", epilogue="sigmoid")
        d = cc.make_desc(dA_, dB_, Y, 1.0, 0.0, precision="bf16x3", epilogue="sigmoid")
        need = C.c_size_t(0)
        assert cc.lib().cucosma_gemm_backward_workspace_size(C.byref(d), C.byref(need)) == cc.SUCCESS
        guard = 1 << 20
        buf = torch.full((need.value + guard,), 0x5A, dtype=torch.uint8, device="cuda")
        gA = to_dev(np.zeros((m, k), np.float32))
        gB = to_dev(np.zeros((k, n), np.float32))
        cc.gemm_backward(dA_, dB_, Y, dY, gA, gB, precision="bf16x3", epilogue="sigmoid",
                         workspace=buf[: need.value])
        torch.cuda.synchronize()
        assert bool((buf[need.value:] == 0x5A).all()), "backward wrote past the queried workspace"
        Yh = Y.cpu().numpy().astype(np.float64)
        G = W.astype(np.float64) * Yh * (1 - Yh)
        refA, refB = oracle.gemm(G, B.T.astype(np.float64)), oracle.gemm(A.T.astype(np.float64), G)
        assert np.abs(gA.cpu().numpy() - refA).max() <= 2e-4 * np.abs(refA).max()
        assert np.abs(gB.cpu().numpy() - refB).max() <= 2e-4 * np.abs(refB).max()
    finally:
        cc.tune_cache_clear()
