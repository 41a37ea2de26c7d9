"""Skinny shapes on the native path (tiny K, or tiny M or N): routing to the
small-K and thin kernels, parity with the FP64 oracle under the rigorous
bound (all alpha/beta/epilogue/dtype combinations, both kernel choices),
split-K determinism, and the reference's special benchmark shapes at full
size (Benchmarks/TESTS_TO_RUN/special.csv: 4 x 8 x 3,000,000 with
SPLIT_K = 320, 4 x 3,000,000 x 4, 38416 x 38416 x 4, 128^3)."""
import numpy as np
import pytest

import cucosma_b200 as cc
import oracle
from tests._util import U32, check_against_oracle, to_dev, uniform

pytestmark = pytest.mark.gpu

SMALL = [(1, 1, 1), (3, 5, 2), (31, 257, 16), (300, 1030, 3), (1, 4000, 9), (2000, 3, 7),  # K <= 16
         (1, 1, 17), (8, 8, 5000), (4, 8, 3001), (7, 300, 700), (9, 8, 513), (1000, 5, 100), (8, 1030, 64)]


def run(A, B, Cin, alpha, beta, dtype, **kw):
    import torch

    dA, dB, dC = to_dev(A.astype(dtype)), to_dev(B.astype(dtype)), to_dev(Cin.astype(dtype))
    d = cc.make_desc(dA, dB, dC, alpha, beta, **{k: v for k, v in kw.items() if k != "workspace"})
    plan = cc.get_plan(d)
    cc.gemm(dA, dB, dC, alpha, beta, **kw)
    torch.cuda.synchronize()
    return dC.cpu().numpy(), plan


@pytest.mark.parametrize("tile", [0, 1], ids=["skinny", "tilekernel"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("shape", SMALL, ids=["%dx%dx%d" % s for s in SMALL])
def test_skinny_vs_oracle(cuda, shape, dtype, tile):
    m, n, k = shape
    A, B, Cin = uniform(1, (m, k), dtype), uniform(2, (k, n), dtype), uniform(3, (m, n), dtype)
    out, plan = run(A, B, Cin, 1.25, -0.5, dtype, tile=tile)
    if tile == 0:
        # skinny kernels: 8 or 64 rows; otherwise the tile kernel (64 or 128 rows for FP32, 128 for FP64)
        want = ((8 if m <= 8 else 64),) if k <= 16 else (8,) if min(m, n) <= 8 else \
            (64, 128) if dtype == np.float32 else (128,)
        assert plan["tile_m"] in want, plan
    check_against_oracle(out, A, B, Cin, 1.25, -0.5, oracle.EPI_NONE, dtype)


@pytest.mark.parametrize("epi,code", [("sigmoid", oracle.EPI_SIGMOID), ("relu", oracle.EPI_RELU)])
@pytest.mark.parametrize("shape", [(300, 1030, 3), (5, 700, 900)], ids=["smallk", "thin"])
def test_skinny_epilogues(cuda, shape, epi, code):
    m, n, k = shape
    A, B, Cin = uniform(4, (m, k)), uniform(5, (k, n)), uniform(6, (m, n))
    out, _ = run(A, B, Cin, 1.0, 0.5, np.float32, epilogue=epi)
    check_against_oracle(out, A, B, Cin, 1.0, 0.5, code, np.float32)


@pytest.mark.parametrize("dtype", [np.float32, np.float64], ids=["f32", "f64"])
def test_thin_forced_split_k_is_deterministic(cuda, dtype):
    m, n, k = 4, 8, 40000
    A, B, Cin = uniform(7, (m, k), dtype), uniform(8, (k, n), dtype), uniform(9, (m, n), dtype)
    out1, plan = run(A, B, Cin, 1.0, 0.5, dtype, split_k=37)
    out2, _ = run(A, B, Cin, 1.0, 0.5, dtype, split_k=37)
    assert plan["splits"] == 37 and plan["workspace_bytes"] > 0
    assert np.array_equal(out1, out2)
    check_against_oracle(out1, A, B, Cin, 1.0, 0.5, oracle.EPI_NONE, dtype)


SPECIAL = [(4, 8, 3_000_000, 320), (4, 3_000_000, 4, 1), (38416, 38416, 4, 1), (128, 128, 128, 4)]


@pytest.mark.slow
@pytest.mark.parametrize("shape", SPECIAL, ids=["%dx%dx%d_sk%d" % s for s in SPECIAL])
def test_reference_special_shapes(cuda, shape):
    """The reference's special rows at full size: checked on sampled rows
    against an FP64 product within the rigorous bound (doubled for the check
    product's own rounding); times of the skinny kernel and of the 128 x 128
    tile kernel are printed."""
    import torch

    m, n, k, sk = shape
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    A = torch.rand((m, k), generator=g, device="cuda") * 2 - 1
    B = torch.rand((k, n), generator=g, device="cuda") * 2 - 1
    C = torch.empty((m, n), device="cuda")
    times = {}
    # (tile id, split_k): the skinny kernel with the reference's SPLIT_K and
    # with the library's choice, then the 128 x 128 tile kernel
    for key in ((0, sk), (0, 0), (1, sk)):
        tile, s_k = key
        s_k = s_k if s_k > 1 else 0
        d = cc.make_desc(A, B, C, split_k=s_k, tile=tile)
        ws = cc.alloc_workspace(d)
        for _ in range(2):
            cc.gemm(A, B, C, split_k=s_k, tile=tile, workspace=ws)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            cc.gemm(A, B, C, split_k=s_k, tile=tile, workspace=ws)
        e1.record()
        torch.cuda.synchronize()
        times[key] = e0.elapsed_time(e1) / 3
        idx = np.unique(np.linspace(0, m - 1, min(m, 8)).astype(np.int64))
        Ah = A[idx].double().cpu().numpy()
        Bh = B.double().cpu().numpy()
        ref = Ah @ Bh
        bnd = 2 * ((k + 2) * U32 * (np.abs(Ah) @ np.abs(Bh)) + 2 * U32 * np.abs(ref))
        out = C[torch.as_tensor(idx, device="cuda")].double().cpu().numpy()
        assert np.all(np.abs(out - ref) <= bnd + 1e-300)
    t_best = min(times[(0, sk)], times[(0, 0)])
    print("%dx%dx%d: skinny %.3f ms with SPLIT_K %d, %.3f ms with the library's split (%.1f GB/s of A+B+C), "
          "tile kernel %.3f ms" % (m, n, k, times[(0, sk)], sk, times[(0, 0)],
                                   4 * (m * k + k * n + m * n) / t_best / 1e6, times[(1, sk)]))
