"""GPU tests of the grouped launch: many uneven GEMMs in one persistent
tcgen05 launch through the C ABI.  Each problem's result is checked bit for
bit against the same precision path launched on its own (same kernel
configuration: 128 x 128 promoted BF16 tiles, no split-K), against the FP64
oracle (BF16 bound, or the bit-exact Ozaki restatement), and the launch is
replayed from a captured CUDA graph."""
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


def shapes(seed, count, lo=1, hi=300, klo=1, khi=500):
    r = np.random.default_rng(seed)
    lu = lambda a, b: int(np.exp(r.uniform(np.log(a), np.log(b))))  # noqa: E731
    return [(lu(lo, hi), lu(lo, hi), lu(klo, khi)) for _ in range(count)]


def make(prob_shapes, dtype, seed):
    host, dev = [], []
    for i, (m, n, k) in enumerate(prob_shapes):
        A = uniform(seed + 3 * i, (m, k), dtype)
        B = uniform(seed + 3 * i + 1, (k, n), dtype)
        Cin = uniform(seed + 3 * i + 2, (m, n), dtype)
        host.append((A, B, Cin))
        dev.append((to_dev(A), to_dev(B), to_dev(Cin)))
    return host, dev


def single(A, B, Cin, precision, slices, alpha, beta):
    """The same path launched on its own, in the grouped kernel's configuration."""
    import torch

    dA, dB, dC = to_dev(A), to_dev(B), to_dev(Cin)
    # grouped tile 1 = the 128 x 128 tiles (BF16x3 promoted: single tile 2; BF16x6: single tile 1)
    tile = 2 if precision == "bf16x3" else 1 if precision == "bf16x6" else 0
    cc.gemm(dA, dB, dC, alpha, beta, precision=precision, slices=slices, split_k=1, tile=tile)
    torch.cuda.synchronize()
    return dC.cpu().numpy()


@pytest.mark.parametrize("precision,dtype,slices", [("bf16x3", np.float32, 0), ("bf16x6", np.float32, 0),
                                                    ("ozaki", np.float64, 8), ("ozaki", np.float64, 6)])
def test_grouped_matches_single_launches(precision, dtype, slices):
    import torch

    sh = shapes(1, 37) + [(1, 1, 1), (128, 128, 32), (129, 257, 33)]
    host, dev = make(sh, dtype, 100)
    plan = cc.grouped(dev, precision=precision, alpha=1.25, beta=0.5, slices=slices)
    plan()
    torch.cuda.synchronize()
    for (A, B, Cin), (_, _, dC) in zip(host, dev):
        out = dC.cpu().numpy()
        ref = single(A, B, Cin, precision, slices, 1.25, 0.5)
        assert np.array_equal(out, ref), (A.shape, B.shape)
        if precision == "ozaki":
            assert np.array_equal(out, oracle.ozaki_gemm(A, B, slices, Cin=Cin, alpha=1.25, beta=0.5))
        else:
            k = A.shape[1]
            u = 2.0 ** -24
            c_split = 3.1 * 2.0 ** -16 if precision == "bf16x3" else 6 * u
            ref64 = oracle.gemm(A, B, Cin, 1.25, 0.5)
            bnd = (c_split + 6 * (k + 2) * u) * 1.25 * oracle.gemm(np.abs(A), np.abs(B)) + 2 * u * (
                np.abs(ref64) + 0.5 * np.abs(Cin)) + 1e-30
            assert np.all(np.abs(out - ref64) <= bnd)


def test_grouped_epilogue_and_beta_zero():
    import torch

    sh = shapes(2, 9)
    host, dev = make(sh, np.float32, 300)
    for _, _, dC in dev:
        dC.fill_(float("nan"))  # beta == 0: C must not be read
    plan = cc.grouped(dev, precision="bf16x6", alpha=1.0, beta=0.0, epilogue="sigmoid")
    plan()
    torch.cuda.synchronize()
    for (A, B, _), (_, _, dC) in zip(host, dev):
        out = dC.cpu().numpy()
        ref = oracle.gemm(A, B, None, 1.0, 0.0, oracle.EPI_SIGMOID)
        assert np.all(np.abs(out - ref) <= 1e-5)


@pytest.mark.parametrize("precision,dtype,slices", [("bf16x3", np.float32, 0), ("ozaki", np.float64, 8)])
def test_grouped_graph_replay(precision, dtype, slices):
    """Capture the grouped launch in a CUDA graph, change the inputs in place,
    replay, and compare with an eager launch on the new inputs."""
    import torch

    sh = shapes(3, 24)
    host, dev = make(sh, dtype, 500)
    plan = cc.grouped(dev, precision=precision, slices=slices)
    plan()  # warm-up outside capture (first launch sets kernel attributes)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            plan(stream=s)
    for (A, B, _), (dA, dB, _) in zip(host, dev):
        dA.mul_(-0.5)
        dB.add_(0.25)
    g.replay()
    torch.cuda.synchronize()
    got = [dC.cpu().numpy().copy() for _, _, dC in dev]
    plan()
    torch.cuda.synchronize()
    for gg, (_, _, dC) in zip(got, dev):
        assert np.array_equal(gg, dC.cpu().numpy())
    n0 = cc.launch_count()
    plan()
    torch.cuda.synchronize()
    assert cc.launch_count() - n0 == (2 if precision != "ozaki" else 3)


def test_grouped_large_batch_matches_single_launches():
    """The benchmark's distribution (M, N log-uniform in [64, 2048], K in
    [64, 8192]) on a subset of 48 problems, GPU against GPU bit for bit."""
    import torch

    sh = shapes(4, 48, 64, 2048, 64, 8192)

    def rand_rows(g, rows, cols):  # 16-byte aligned rows
        buf = torch.rand((rows, -(-cols // 4) * 4), generator=g, device="cuda") * 2 - 1
        return buf[:, :cols]

    dev = []
    for i, (m, n, k) in enumerate(sh):
        g = torch.Generator(device="cuda")
        g.manual_seed(1000 + i)
        dev.append((rand_rows(g, m, k), rand_rows(g, k, n), torch.zeros((m, -(-n // 4) * 4), device="cuda")[:, :n]))
    plan = cc.grouped(dev, precision="bf16x3")
    plan()
    torch.cuda.synchronize()
    for A, B, Cm in dev[:12]:
        ref = torch.zeros((Cm.shape[0], Cm.stride(0)), device="cuda")[:, :Cm.shape[1]]
        cc.gemm(A, B, ref, precision="bf16x3", split_k=1, tile=2)
        torch.cuda.synchronize()
        assert torch.equal(ref, Cm)


def test_grouped_rejects_bad_input():
    import ctypes as C

    L = cc.lib()
    d = cc.GemmDesc()
    L.cucosma_gemm_desc_init(C.byref(d))
    d.precision = cc.PRECISIONS["native"]
    arr = (cc._ext.Problem * 1)()
    arr[0] = cc._ext.Problem(8, 8, 8, 8, 8, 8, 0x10000, 0x10000, 0x10000)
    n = C.c_size_t(0)
    assert L.cucosma_grouped_workspace_size(C.byref(d), arr, 1, C.byref(n)) == cc.NOT_SUPPORTED
    d.precision = cc.PRECISIONS["bf16x3"]
    assert L.cucosma_grouped_workspace_size(C.byref(d), arr, 1, C.byref(n)) == cc.SUCCESS
    arr[0] = cc._ext.Problem(8, 8, 8, 9, 8, 8, 0x10000, 0x10000, 0x10000)
    assert L.cucosma_grouped_workspace_size(C.byref(d), arr, 1, C.byref(n)) == cc.MISALIGNED
    assert L.cucosma_grouped_workspace_size(C.byref(d), arr, 0, C.byref(n)) == cc.INVALID_VALUE


# grouped tile id -> the single-launch tile id with the same per-element arithmetic
GROUPED_TILES = [("bf16x3", 1, 2), ("bf16x3", 2, 3), ("bf16x3", 3, 4), ("bf16x6", 1, 1), ("bf16x6", 2, 3)]


@pytest.mark.parametrize("precision,gtile,stile", GROUPED_TILES,
                         ids=["bf16x3-128x128", "bf16x3-128x256", "bf16x3-pair256", "bf16x6-128x128",
                              "bf16x6-pair256"])
def test_grouped_tiles_match_single_launches(precision, gtile, stile):
    """Every grouped tile (CTA-pair tiles included) gives each problem's
    result bit for bit as the single launch with the same tile."""
    import torch

    sh = shapes(3, 23, hi=700, khi=900) + [(1, 1, 1), (257, 129, 40), (600, 300, 77)]
    host, dev = make(sh, np.float32, 300)
    plan = cc.grouped(dev, precision=precision, alpha=1.0, beta=0.5, tile=gtile)
    assert plan.tile()[:1] == (gtile,) and not plan.tile()[3]
    plan()
    torch.cuda.synchronize()
    for (A, B, Cin), (_, _, dC) in zip(host, dev):
        dA, dB, dS = to_dev(A), to_dev(B), to_dev(Cin)
        cc.gemm(dA, dB, dS, 1.0, 0.5, precision=precision, split_k=1, tile=stile)
        torch.cuda.synchronize()
        assert np.array_equal(dC.cpu().numpy(), dS.cpu().numpy()), (A.shape, B.shape)


def test_grouped_plan_takes_its_tile_from_the_tuner():
    """cucosma_tune_grouped measures the grouped tiles on a batch and caches
    the fastest for its shape mix; a plan created afterwards with tile 0 uses
    that tile (reported as coming from the cache), its results equal a plan
    with that tile given explicitly, and the measured L2 hit rate and DRAM
    bytes of the chosen launch are reported."""
    import torch

    cc.tune_cache_clear()
    try:
        sh = shapes(4, 31, lo=64, hi=1024, klo=64, khi=2048)
        _, dev = make(sh, np.float32, 400)
        base = cc.grouped(dev, precision="bf16x3")
        assert base.tile() == (1, 128, 128, False)
        r = base.tune()
        print("grouped tune:", r)
        assert r["candidates"] == 3 and r["tile"] in (1, 2, 3) and r["ms"] > 0
        assert 0.0 <= r["l2_hit_rate"] <= 100.0 and r["dram_bytes"] > 0
        tuned = cc.grouped(dev, precision="bf16x3")
        tid, tm, tn, from_cache = tuned.tile()
        assert from_cache and tid == r["tile"]
        tuned()
        torch.cuda.synchronize()
        got = [d[2].cpu().numpy().copy() for d in dev]
        explicit = cc.grouped(dev, precision="bf16x3", tile=tid)
        explicit()
        torch.cuda.synchronize()
        for g, d in zip(got, dev):
            assert np.array_equal(g, d[2].cpu().numpy())
        # another batch keeps the default tile
        other = cc.grouped(dev[:-1], precision="bf16x3")
        assert other.tile()[3] is False
    finally:
        cc.tune_cache_clear()
