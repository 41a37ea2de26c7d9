"""The autotuner (cucosma_tune) and its cache.  CPU: the cache file format
round-trips without a GPU.  GPU: tuning measures several candidates, records
the fastest, and later auto-configured calls use it and stay correct."""
import os

import numpy as np
import pytest

import cucosma_b200 as cc
import oracle
from tests._util import check_against_oracle, to_dev, uniform

LINES = ["v2 148 0 0 0 1024 1024 1024 3 1 0 0.123000 71.250 12582912",
         "v2 148 0 1 0 8192 8192 8192 1 8 4 2.500000 -1.000 -1"]


def test_cache_file_roundtrip(tmp_path):
    cc.tune_cache_clear()
    src = tmp_path / "in.txt"
    src.write_text("\n".join(LINES) + "\n")
    cc.tune_cache_load(str(src))
    assert cc.tune_cache_size() == 2
    out = tmp_path / "out.txt"
    cc.tune_cache_save(str(out))
    assert sorted(out.read_text().strip().splitlines()) == sorted(LINES)
    cc.tune_cache_clear()
    assert cc.tune_cache_size() == 0


def test_cache_reads_v1_lines(tmp_path):
    """Cache files written before the counter readings (v1 lines) still load;
    their entries carry no measurement (-1)."""
    cc.tune_cache_clear()
    src = tmp_path / "v1.txt"
    src.write_text("v1 148 0 0 0 1024 1024 1024 3 1 0 0.123000\n")
    cc.tune_cache_load(str(src))
    assert cc.tune_cache_size() == 1
    out = tmp_path / "out.txt"
    cc.tune_cache_save(str(out))
    assert out.read_text().strip() == "v2 148 0 0 0 1024 1024 1024 3 1 0 0.123000 -1.000 -1"
    cc.tune_cache_clear()


@pytest.mark.gpu
@pytest.mark.parametrize("precision,dtype", [("native", np.float32), ("bf16x3", np.float32), ("native", np.float64)])
def test_tune_then_use(cuda, tmp_path, precision, dtype):
    import torch

    cc.tune_cache_clear()
    m, n, k = 384, 320, 6000
    A, B = uniform(1, (m, k), dtype), uniform(2, (k, n), dtype)
    Cin = uniform(3, (m, n), dtype)
    dA, dB = to_dev(A), to_dev(B)
    scratch = to_dev(np.zeros((m, n), dtype))
    r = cc.tune(dA, dB, scratch, 1.0, 0.5, precision=precision)
    print(precision, r)
    assert r["candidates"] >= 3 and r["ms"] > 0 and r["tflops"] > 0 and r["occupancy"] >= 1
    # the L2 hit rate and DRAM traffic of the chosen configuration, read from
    # the hardware counters (CUPTI range profiler) on this GPU
    assert 0.0 <= r["l2_hit_rate"] <= 100.0 and r["counter_passes"] >= 1
    assert r["dram_bytes"] > 0
    assert cc.tune_cache_size() == 1
    dC = to_dev(Cin)
    plan = cc.get_plan(cc.make_desc(dA, dB, dC, 1.0, 0.5, precision=precision))
    # a forced split count s becomes ceil(k / kchunk) splits, kchunk = round_up(ceil(k / s), tile_k)
    kchunk = -(-(-(-k // r["split_k"])) // plan["tile_k"]) * plan["tile_k"]
    assert plan["splits"] == min(r["split_k"], -(-k // kchunk))
    if precision == "native":
        # the picked tile id fixes the CTA height: 1 -> 128 rows, 2 -> 64 (FP32)
        assert r["tile"] in ((1, 2) if dtype == np.float32 else (0,))
        if dtype == np.float32:
            assert plan["tile_m"] == (64 if r["tile"] == 2 else 128)
    cc.gemm(dA, dB, dC, 1.0, 0.5, precision=precision)
    torch.cuda.synchronize()
    out = dC.cpu().numpy()
    if precision == "native":
        check_against_oracle(out, A, B, Cin, 1.0, 0.5, oracle.EPI_NONE, dtype)
    else:
        ref = oracle.gemm(A, B, Cin, 1.0, 0.5)
        assert oracle.errors(out, ref)["normwise"] < 1e-4
    path = tmp_path / "cache.txt"
    cc.tune_cache_save(str(path))
    cc.tune_cache_clear()
    cc.tune_cache_load(str(path))
    assert cc.tune_cache_size() == 1
    os.environ["CUCOSMA_TUNE"] = "off"
    try:
        p_off = cc.get_plan(cc.make_desc(dA, dB, dC, 1.0, 0.5, precision=precision))
    finally:
        del os.environ["CUCOSMA_TUNE"]
    p_on = cc.get_plan(cc.make_desc(dA, dB, dC, 1.0, 0.5, precision=precision))
    assert p_on["splits"] == plan["splits"]
    cc.tune_cache_clear()
    assert p_off["splits"] == cc.get_plan(cc.make_desc(dA, dB, dC, 1.0, 0.5, precision=precision))["splits"]


@pytest.mark.gpu
def test_tune_skinny_shape_compares_kernels(cuda):
    """A thin shape: the tuner weighs the skinny kernel (tile 0) against the
    128 x 128 tile kernel (tile 1) and later calls use its pick correctly."""
    import torch

    cc.tune_cache_clear()
    m, n, k = 4, 8, 200000
    A, B = uniform(11, (m, k)), uniform(12, (k, n))
    dA, dB = to_dev(A), to_dev(B)
    scratch = to_dev(np.zeros((m, n), np.float32))
    ws = torch.empty(64 << 20, dtype=torch.uint8, device="cuda")
    r = cc.tune(dA, dB, scratch, 1.0, 0.0, workspace=ws)
    print(r)
    assert r["candidates"] >= 2 and r["tile"] in (0, 1)
    dC = to_dev(np.zeros((m, n), np.float32))
    cc.gemm(dA, dB, dC, 1.0, 0.0, workspace=ws)
    torch.cuda.synchronize()
    check_against_oracle(dC.cpu().numpy(), A, B, np.zeros((m, n), np.float32), 1.0, 0.0, oracle.EPI_NONE,
                         np.float32)
    cc.tune_cache_clear()
