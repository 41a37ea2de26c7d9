"""GPU parity tests of the native FP32 (FFMA) / FP64 (DFMA) path through the
C ABI, against the FP64 oracle (rigorous componentwise bound), the golden
fixtures, and the reference kernel cosmaSgemm built from its own sources
(oracle/_ref, when present)."""
import glob
import os

import numpy as np
import pytest

import cucosma_b200 as cc
import oracle
from tests._util import bound, check_against_oracle, to_dev, uniform

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1, 1), (7, 5, 3), (4, 8, 300), (127, 127, 127), (128, 128, 128), (129, 257, 65), (300, 200, 100),
          (1000, 4, 17), (33, 1000, 5), (512, 384, 1024)]


def run(A, B, Cin, alpha, beta, dtype, epilogue="none", ld_pad=0, **kw):
    import torch

    es = np.dtype(dtype).itemsize
    pad = ld_pad * (16 // es)
    dA = to_dev(A.astype(dtype), ld=None if not pad else A.shape[1] + pad + (-(A.shape[1]) % (16 // es)))
    dB = to_dev(B.astype(dtype), ld=None if not pad else B.shape[1] + pad + (-(B.shape[1]) % (16 // es)))
    dC = to_dev(Cin.astype(dtype))
    cc.gemm(dA, dB, dC, alpha, beta, epilogue=epilogue, **kw)
    torch.cuda.synchronize()
    return dC.cpu().numpy()


@pytest.mark.parametrize("dtype", [np.float32, np.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("shape", SHAPES, ids=["%dx%dx%d" % s for s in SHAPES])
def test_native_vs_oracle(cuda, shape, dtype):
    m, n, k = shape
    A = uniform(1, (m, k), dtype)
    B = uniform(2, (k, n), dtype)
    Cin = uniform(3, (m, n), dtype)
    out = run(A, B, Cin, 1.0, 0.5, dtype)
    check_against_oracle(out, A, B, Cin, 1.0, 0.5, oracle.EPI_NONE, dtype)


@pytest.mark.parametrize("dtype", [np.float32, np.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-1.5, 0.0), (0.75, 1.0), (2.0, -0.5), (0.0, 0.5), (0.0, 0.0)])
def test_alpha_beta(cuda, dtype, alpha, beta):
    A = uniform(4, (200, 150), dtype)
    B = uniform(5, (150, 170), dtype)
    Cin = uniform(6, (200, 170), dtype)
    out = run(A, B, Cin, alpha, beta, dtype)
    check_against_oracle(out, A, B, Cin, alpha, beta, oracle.EPI_NONE, dtype)


def test_beta_zero_ignores_nan_c(cuda):
    A = uniform(7, (64, 64))
    B = uniform(8, (64, 64))
    Cin = np.full((64, 64), np.nan, np.float32)
    out = run(A, B, Cin, 1.0, 0.0, np.float32)
    assert np.isfinite(out).all()


@pytest.mark.parametrize("dtype", [np.float32, np.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("epi", ["sigmoid", "relu"])
def test_fused_epilogue(cuda, dtype, epi):
    A = uniform(9, (257, 130), dtype)
    B = uniform(10, (130, 300), dtype)
    Cin = uniform(11, (257, 300), dtype)
    out = run(A, B, Cin, 1.0, 0.5, dtype, epilogue=epi)
    code = oracle.EPI_SIGMOID if epi == "sigmoid" else oracle.EPI_RELU
    check_against_oracle(out, A, B, Cin, 1.0, 0.5, code, dtype)


@pytest.mark.parametrize("dtype", [np.float32, np.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("split_k", [1, 2, 3, 7, 40])
def test_split_k(cuda, dtype, split_k):
    A = uniform(12, (130, 2000), dtype)
    B = uniform(13, (2000, 129), dtype)
    Cin = uniform(14, (130, 129), dtype)
    out = run(A, B, Cin, 1.0, 0.5, dtype, split_k=split_k)
    check_against_oracle(out, A, B, Cin, 1.0, 0.5, oracle.EPI_NONE, dtype)


def test_split_k_sigmoid(cuda):
    A = uniform(15, (100, 3000))
    B = uniform(16, (3000, 90))
    Cin = uniform(17, (100, 90))
    out = run(A, B, Cin, 0.5, 0.5, np.float32, epilogue="sigmoid", split_k=5)
    check_against_oracle(out, A, B, Cin, 0.5, 0.5, oracle.EPI_SIGMOID, np.float32)


@pytest.mark.parametrize("swizzle", [2, 3, 4, 8])
def test_swizzle(cuda, swizzle):
    A = uniform(18, (1000, 64))
    B = uniform(19, (64, 700))
    Cin = uniform(20, (1000, 700))
    out = run(A, B, Cin, 1.0, 0.5, np.float32, swizzle=swizzle)
    check_against_oracle(out, A, B, Cin, 1.0, 0.5, oracle.EPI_NONE, np.float32)


def test_padded_leading_dimensions(cuda):
    A = uniform(21, (77, 93))
    B = uniform(22, (93, 61))
    Cin = uniform(23, (77, 61))
    out = run(A, B, Cin, 1.0, 0.5, np.float32, ld_pad=3)
    check_against_oracle(out, A, B, Cin, 1.0, 0.5, oracle.EPI_NONE, np.float32)


@pytest.mark.parametrize("dtype", [np.float32, np.float64], ids=["f32", "f64"])
def test_deterministic_bitwise(cuda, dtype):
    A = uniform(24, (300, 5000), dtype)
    B = uniform(25, (5000, 200), dtype)
    Cin = uniform(26, (300, 200), dtype)
    outs = [run(A, B, Cin, 1.0, 0.5, dtype, split_k=6) for _ in range(3)]
    assert all(np.array_equal(outs[0], o) for o in outs[1:])


# The 64 x 128 CTA tile (tile id 2, FP32): partial tiles in both directions,
# K below and above one stage, split-K, the fused epilogue and padded rows.
TILE64 = [(1, 1, 1), (63, 129, 17), (64, 128, 16), (65, 300, 1000), (200, 70, 3), (513, 257, 700)]


@pytest.mark.parametrize("split_k", [0, 3])
@pytest.mark.parametrize("shape", TILE64, ids=["%dx%dx%d" % s for s in TILE64])
def test_tile64_vs_oracle(cuda, shape, split_k):
    m, n, k = shape
    A, B, Cin = uniform(40, (m, k)), uniform(41, (k, n)), uniform(42, (m, n))
    out = run(A, B, Cin, 1.25, 0.5, np.float32, tile=2, split_k=split_k)
    check_against_oracle(out, A, B, Cin, 1.25, 0.5, oracle.EPI_NONE, np.float32)


def test_tile64_sigmoid_padded(cuda):
    A, B, Cin = uniform(43, (150, 301)), uniform(44, (301, 77)), uniform(45, (150, 77))
    out = run(A, B, Cin, 1.0, 0.5, np.float32, epilogue="sigmoid", ld_pad=2, tile=2)
    check_against_oracle(out, A, B, Cin, 1.0, 0.5, oracle.EPI_SIGMOID, np.float32)


@pytest.mark.parametrize("split_k", [1, 4])
def test_tile64_bitwise_equal_to_tile128(cuda, split_k):
    """Both CTA heights accumulate every output over k in the same order
    (ascending, one fmaf per k, splits added in order), so they agree bit for bit."""
    A, B, Cin = uniform(46, (333, 2000)), uniform(47, (2000, 260)), uniform(48, (333, 260))
    o128 = run(A, B, Cin, 1.0, 0.5, np.float32, tile=1, split_k=split_k)
    o64 = run(A, B, Cin, 1.0, 0.5, np.float32, tile=2, split_k=split_k)
    assert np.array_equal(o128, o64)


def test_tile_ids_in_plan(cuda):
    import torch

    for dtype, want in ((torch.float32, 64), (torch.float64, 128)):
        A = torch.zeros((300, 200), dtype=dtype, device="cuda")
        B = torch.zeros((200, 500), dtype=dtype, device="cuda")
        Cm = torch.zeros((300, 500), dtype=dtype, device="cuda")
        assert cc.get_plan(cc.make_desc(A, B, Cm, tile=2))["tile_m"] == want
        assert cc.get_plan(cc.make_desc(A, B, Cm, tile=1))["tile_m"] == 128


def test_reference_entry_point_concurrent_streams(cuda):
    """cucosma_sgemm's library-managed split-K workspace is per stream: two
    split-K calls queued on two streams without any ordering between them
    must both come out right (a shared workspace would mix their partials)."""
    import torch

    m, n, k = 100, 90, 30000
    assert cc.get_plan(cc.make_desc(to_dev(np.zeros((m, k), np.float32)), to_dev(np.zeros((k, n), np.float32)),
                                    to_dev(np.zeros((m, n), np.float32))))["splits"] > 1
    cases = []
    for seed in (60, 70):
        A, B, Cin = uniform(seed, (m, k)), uniform(seed + 1, (k, n)), uniform(seed + 2, (m, n))
        cases.append((A, B, Cin, to_dev(A), to_dev(B), to_dev(Cin)))
    torch.cuda.synchronize()
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    for rep in range(3):
        for (A, B, Cin, dA, dB, dC), st in zip(cases, streams):
            with torch.cuda.stream(st):
                cc.cosma_sgemm(dA, dB, dC, 1.0, 0.0 if rep else 0.5, stream=st)
    torch.cuda.synchronize()
    for A, B, Cin, dA, dB, dC in cases:
        check_against_oracle(dC.cpu().numpy(), A, B, Cin, 1.0, 0.0, oracle.EPI_NONE, np.float32)


GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "gemm_*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_golden_fixtures(cuda, path):
    g = np.load(path)
    A, B = g["A"], g["B"]
    Cin = np.zeros((A.shape[0], B.shape[1]), np.float32)
    out = run(A, B, Cin, 1.0, 0.0, np.float32)
    k = A.shape[1]
    absab = oracle.gemm(np.abs(A), np.abs(B))
    assert np.all(np.abs(out - g["prod_f64"]) <= (k + 2) * 2.0 ** -24 * absab + 1e-30)


def test_reference_shaped_entry_point(cuda):
    import torch

    for dtype in (np.float32, np.float64):
        A = uniform(27, (150, 80), dtype)
        B = uniform(28, (80, 140), dtype)
        Cin = uniform(29, (150, 140), dtype)
        dA, dB, dC = to_dev(A), to_dev(B), to_dev(Cin)
        cc.cosma_sgemm(dA, dB, dC, 1.0, 0.5)
        torch.cuda.synchronize()
        check_against_oracle(dC.cpu().numpy(), A, B, Cin, 1.0, 0.5, oracle.EPI_NONE, dtype)


def test_device_status_clean_after_runs(cuda):
    s, code = cc.device_status()
    assert s == cc.SUCCESS and code == 0


# --------------------------------------------------------- reference kernel


REF_TAGS = [t for t in oracle.ref_kernel_tags() if "8192" not in t]


@pytest.mark.parametrize("tag", REF_TAGS)
def test_parity_with_reference_kernel(cuda, tag):
    """Same seeded inputs through the reference kernel (compiled unmodified for
    sm_100a) and through this library: both inside the FP64-oracle bound, and
    their difference from each other stated and bounded -- entrywise by the
    sum of the two bounds (each is within its bound of the oracle), and
    normwise by twice the larger of their two normwise errors plus u."""
    import torch

    ref = oracle.RefKernel(tag)
    c = ref.config
    dtype = np.float32 if c["elem"] == 4 else np.float64
    m, n, k = c["m"], c["n"], c["k"]
    A = uniform(31, (m, k), dtype)
    B = uniform(32, (k, n), dtype)
    Cin = uniform(33, (m, n), dtype)
    pitch = 512 // np.dtype(dtype).itemsize  # cudaMallocPitch-like rows
    ld = lambda cols: -(-cols // pitch) * pitch  # noqa: E731
    rA, rB, rC = to_dev(A, ld(k)), to_dev(B, ld(n)), to_dev(Cin, ld(n))
    rc = ref(rA.data_ptr(), rA.stride(0), rB.data_ptr(), rB.stride(0), rC.data_ptr(), rC.stride(0))
    torch.cuda.synchronize()
    assert rc == 0
    out_ref = rC.cpu().numpy()
    out = run(A, B, Cin, ref.alpha, ref.beta, dtype)
    e_ref = check_against_oracle(out_ref, A, B, Cin, ref.alpha, ref.beta, oracle.EPI_NONE, dtype)
    e_own = check_against_oracle(out, A, B, Cin, ref.alpha, ref.beta, oracle.EPI_NONE, dtype)
    # ours against the reference's own result on the same inputs
    e_pair = oracle.errors(out, out_ref.astype(np.float64))
    pre = oracle.gemm(A, B, Cin, ref.alpha, ref.beta)
    b = bound(A, B, Cin, ref.alpha, ref.beta, oracle.EPI_NONE, dtype, pre)
    diff = np.abs(out.astype(np.float64) - out_ref.astype(np.float64))
    u = 2.0 ** -24 if dtype == np.float32 else 2.0 ** -53
    print(tag, "reference", e_ref, "cucosma", e_own, "cucosma vs reference", e_pair)
    assert np.all(diff <= 2 * b)
    assert e_pair["normwise"] <= 2 * max(e_ref["normwise"], e_own["normwise"]) + u
