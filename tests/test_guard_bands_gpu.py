"""Guard bands: every path writes only the M x N region of C.  C sits inside
a larger buffer (extra columns beyond N in each padded row, extra rows above
and below) filled with a sentinel; after the call the sentinel must be
intact everywhere outside the region, and the region itself must be
finite.  Stands in for a memory checker (compute-sanitizer is not used
here) on the paths and shapes with partial tiles, split-K and the skinny
kernels."""
import numpy as np
import pytest

import cucosma_b200 as cc
from tests._util import to_dev, uniform

pytestmark = pytest.mark.gpu

SENTINEL = 1234.5

CASES = [  # (precision, dtype, m, n, k, split_k[, tile])
    ("native", np.float32, 130, 67, 45, 0), ("native", np.float32, 300, 200, 3000, 3),
    ("native", np.float64, 129, 257, 65, 0), ("native", np.float64, 77, 61, 900, 5),
    ("native", np.float32, 300, 1030, 3, 0), ("native", np.float32, 4, 9, 5000, 0),
    ("native", np.float64, 1000, 5, 100, 0), ("native", np.float32, 6, 700, 900, 7),
    ("bf16x3", np.float32, 129, 257, 65, 0), ("bf16x3", np.float32, 200, 300, 3000, 2),
    ("bf16x6", np.float32, 130, 70, 45, 0), ("ozaki", np.float64, 129, 65, 33, 0),
    ("ozaki", np.float64, 70, 90, 3000, 3),
    ("native", np.float32, 130, 67, 45, 0, 2), ("native", np.float32, 65, 300, 3000, 3, 2),
    # N a multiple of 4: C leaves through TMA boxes (partial tiles right and below)
    ("bf16x3", np.float32, 129, 260, 65, 0), ("bf16x6", np.float32, 130, 72, 45, 0),
    ("bf16x3", np.float32, 300, 132, 3000, 0, 5), ("bf16x6", np.float32, 300, 132, 3000, 0, 4),
    # N a multiple of 32 with an odd number of 32-column chunks: 64-column 3-D boxes, the last half outside
    ("bf16x3", np.float32, 129, 96, 65, 0), ("bf16x6", np.float32, 260, 160, 45, 0),
    # FP64 with N even: the Ozaki results leave through 32 x 16 TMA boxes
    ("ozaki", np.float64, 129, 66, 33, 0), ("ozaki", np.float64, 300, 130, 700, 0),
]


@pytest.mark.parametrize("case", CASES, ids=["%s_%s_%dx%dx%d_sk%d" % (c[0], np.dtype(c[1]).name, *c[2:6])
                                             + ("_t%d" % c[6] if len(c) > 6 else "") for c in CASES])
def test_writes_stay_inside_c(cuda, case):
    import torch

    prec, dtype, m, n, k, split_k = case[:6]
    tile = case[6] if len(case) > 6 else 0
    es = np.dtype(dtype).itemsize
    A, B = uniform(1, (m, k), dtype), uniform(2, (k, n), dtype)
    dA, dB = to_dev(A), to_dev(B)
    vec = 16 // es
    ld = -(-n // vec) * vec + 2 * vec  # two 16-byte groups of padding per row
    tdt = torch.float32 if dtype == np.float32 else torch.float64
    buf = torch.full((m + 4, ld), SENTINEL, dtype=tdt, device="cuda")
    C = buf[2:2 + m, :n]
    C.zero_()
    cc.gemm(dA, dB, C, 1.0, 0.0, precision=prec, split_k=split_k, tile=tile)
    torch.cuda.synchronize()
    h = buf.cpu().numpy()
    region = np.zeros(h.shape, bool)
    region[2:2 + m, :n] = True
    assert np.all(h[~region] == SENTINEL), "a write landed outside C"
    assert np.all(np.isfinite(h[region]))
    assert cc.device_status() == (cc.SUCCESS, 0)
