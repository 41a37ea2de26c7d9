"""Full-size parity of the reference's benchmark shape families through the C
ABI: square 8192^3, flat 16384 x 16384 x 256, large-K 256 x 256 x 1,048,576
(split-K) and large-N 256 x 1,048,576 x 256, FP32 and FP64 native
arithmetic, alpha = 1, beta = 0.5, C uniform[-1, 1], with and without the
sigmoid epilogue.  Results are checked on 8 sampled rows against an FP64
product within the rigorous bound (doubled: the check product has its own
FP64 rounding), and the time of each call is printed."""
import numpy as np
import pytest

import cucosma_b200 as cc

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

FAMILIES = {"SQ": (8192, 8192, 8192), "FL": (16384, 16384, 256), "LK": (256, 256, 1 << 20),
            "LN": (256, 1 << 20, 256)}


def rand(shape, dtype, seed):
    import torch

    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    return torch.rand(shape, generator=g, device="cuda", dtype=dtype) * 2 - 1


@pytest.mark.parametrize("epilogue", ["none", "sigmoid"])
@pytest.mark.parametrize("dtype_name", ["f32", "f64"])
@pytest.mark.parametrize("family", list(FAMILIES))
def test_family(cuda, family, dtype_name, epilogue):
    import torch

    dtype = torch.float32 if dtype_name == "f32" else torch.float64
    m, n, k = FAMILIES[family]
    A, B, C0 = rand((m, k), dtype, 1), rand((k, n), dtype, 2), rand((m, n), dtype, 3)
    Cm = C0.clone()
    cc.gemm(A, B, Cm, 1.0, 0.5, epilogue=epilogue)
    torch.cuda.synchronize()
    # time a few more calls (C is overwritten; the values are not re-checked)
    Ct = C0.clone()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(3):
        cc.gemm(A, B, Ct, 1.0, 0.5, epilogue=epilogue)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 3
    plan = cc.get_plan(cc.make_desc(A, B, Cm, 1.0, 0.5, epilogue=epilogue))
    print("%s %s %s: %.3f ms, %.2f TFLOP/s, splits %d" % (family, dtype_name, epilogue, ms, 2.0 * m * n * k / ms / 1e9,
                                                           plan["splits"]))
    idx = np.linspace(0, m - 1, 8).astype(np.int64)
    Ah = A[idx].double().cpu().numpy()
    Bh = B.double().cpu().numpy()
    Ch = C0[idx].double().cpu().numpy()
    pre = Ah @ Bh + 0.5 * Ch
    ref = 1.0 / (1.0 + np.exp(-pre)) if epilogue == "sigmoid" else pre
    u = 2.0 ** -24 if dtype == torch.float32 else 2.0 ** -53
    bound = 2 * ((k + 2) * u * (np.abs(Ah) @ np.abs(Bh)) + 2 * u * (np.abs(pre) + 0.5 * np.abs(Ch)))
    if epilogue == "sigmoid":
        bound = 0.25 * bound + 8 * u
    out = Cm[idx].double().cpu().numpy()
    err = np.abs(out - ref)
    assert np.all(err <= bound + 1e-300), float((err / (bound + 1e-300)).max())
