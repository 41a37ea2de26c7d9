"""CPU tests of the oracle: pinned against the reference's own code and the
committed golden fixtures, plus the algebraic properties of the BF16 split
and Ozaki restatements.  No GPU needed."""
import glob
import os
from fractions import Fraction

import numpy as np
import pytest

import oracle
from tests._util import uniform, expspread

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "gemm_*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_oracle_bitexact_vs_golden(path):
    g = np.load(path)
    out = oracle.gemm(g["A"], g["B"])
    # Same i-j-k order, double accumulation, no contraction: bit for bit.
    assert np.array_equal(out, g["prod_f64"])
    # The reference's float-accumulating CPU product stays within the float bound.
    k = g["A"].shape[1]
    absab = oracle.gemm(np.abs(g["A"]), np.abs(g["B"]))
    assert np.all(np.abs(g["prod_f32"] - out) <= k * 2.0 ** -24 * absab * 1.01 + 1e-30)


def test_golden_fixtures_present():
    assert len(GOLDEN) >= 5


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("shape", [(1, 1, 1), (5, 3, 7), (37, 29, 53), (64, 48, 200)])
def test_oracle_bitexact_vs_reference_cpu(shape):
    m, n, k = shape
    A = uniform(11, (m, k), np.float64)
    B = uniform(12, (k, n), np.float64)
    assert np.array_equal(oracle.gemm(A, B), oracle.ref_product(A, B))


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
def test_reference_generator_matches_fixture():
    g = np.load(GOLDEN[0])
    m, k = g["A"].shape
    sa = int(g["seeds"][0])
    assert np.array_equal(oracle.ref_fill_random(sa, m, k, np.float32), g["A"])


def test_alpha_beta_epilogue_semantics():
    A = uniform(1, (9, 13), np.float64)
    B = uniform(2, (13, 7), np.float64)
    Cin = uniform(3, (9, 7), np.float64)
    out = oracle.gemm(A, B, Cin, alpha=1.5, beta=-0.25)
    np.testing.assert_allclose(out, 1.5 * (A @ B) - 0.25 * Cin, rtol=1e-13, atol=1e-13)
    sig = oracle.gemm(A, B, Cin, 1.5, -0.25, oracle.EPI_SIGMOID)
    np.testing.assert_allclose(sig, 1 / (1 + np.exp(-out)), rtol=1e-14)
    relu = oracle.gemm(A, B, Cin, 1.5, -0.25, oracle.EPI_RELU)
    np.testing.assert_array_equal(relu, np.maximum(out, 0))
    # beta == 0 never reads C: NaNs in C must not leak.
    nanC = np.full((9, 7), np.nan)
    assert np.isfinite(oracle.gemm(A, B, nanC, 1.0, 0.0)).all()


def test_double_double_exact_on_small_case():
    A = uniform(4, (3, 50), np.float64)
    B = uniform(5, (50, 2), np.float64)
    hi, lo = oracle.gemm(A, B, dd=True)
    for i in range(3):
        for j in range(2):
            exact = sum(Fraction(float(A[i, k])) * Fraction(float(B[k, j])) for k in range(50))
            assert abs(Fraction(hi[i, j]) + Fraction(lo[i, j]) - exact) <= abs(exact) * Fraction(1, 2 ** 100)


def test_splitk_reduce_restatement_order():
    ws = uniform(6, (3, 4, 5), np.float32)
    Cin = uniform(7, (4, 5), np.float32)
    out = oracle.splitk_reduce_f32(ws, Cin, np.float32(1.0), np.float32(0.5))
    s = (ws[0] + ws[1]) + ws[2]
    np.testing.assert_array_equal(out, np.float32(0.5) * Cin + np.float32(1.0) * s)


@pytest.mark.parametrize("nterms", [1, 2, 3])
def test_bf16_split_residual_bound(nterms):
    x = np.concatenate([uniform(8, (4000,)), expspread(9, (4000,), 4.0, np.float32)]).astype(np.float32)
    t = oracle.split_bf16(x, nterms)
    rec = sum(oracle.bf16_to_f32(t[i]).astype(np.float64) for i in range(nterms))
    err = np.abs(rec - x.astype(np.float64))
    # BF16 keeps 8 significant bits: each round-to-nearest term leaves a
    # residual of at most 2^-8 of what it rounded
    assert np.all(err <= np.abs(x) * 2.0 ** (-8 * nterms) * 1.0000001)
    if nterms == 3:
        assert np.array_equal(rec.astype(np.float32), x)


def test_bf16_split_hi_is_round_to_nearest_even():
    x = np.array([1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -1.0 - 2 ** -8, 3.0], np.float32)
    hi = oracle.bf16_to_f32(oracle.split_bf16(x, 1)[0])
    np.testing.assert_array_equal(hi, np.array([1.0, 1.0 + 2 ** -6, -1.0, 3.0], np.float32))


@pytest.mark.parametrize("dist", ["uniform", "expspread"])
def test_ozaki_slices_reconstruct(dist):
    A = uniform(10, (17, 40), np.float64) if dist == "uniform" else expspread(10, (17, 40))
    B = uniform(11, (40, 13), np.float64) if dist == "uniform" else expspread(11, (40, 13))
    s = 8
    ea, eb, sa, sb = oracle.ozaki_slices(A, B, s)
    assert sa.dtype == np.int8 and np.abs(sa.astype(int)).max() <= 127
    w = 2.0 ** (-7 * (np.arange(s) + 1))
    recA = np.tensordot(w, sa.astype(np.float64), 1) * 2.0 ** ea[:, None]
    recB = (np.tensordot(w, sb.astype(np.float64), 1) * 2.0 ** eb[:, None]).T
    # residual below 2^-7s of the row / column scale
    assert np.all(np.abs(recA - A) <= 2.0 ** (ea[:, None] - 7 * s))
    assert np.all(np.abs(recB - B) <= 2.0 ** (eb[None, :] - 7 * s))
    # every row max sits in [2^(e-1), 2^e)
    mx = np.abs(A).max(axis=1)
    assert np.all((mx < 2.0 ** ea) & (mx >= 2.0 ** (ea - 1)))


def test_ozaki_error_decreases_with_slices():
    A = uniform(12, (48, 300), np.float64)
    B = uniform(13, (300, 40), np.float64)
    hi, lo = oracle.gemm(A, B, dd=True)
    errs = [oracle.errors(oracle.ozaki_gemm(A, B, s), hi, lo)["normwise"] for s in (4, 5, 6, 7, 8)]
    assert all(a > b for a, b in zip(errs, errs[1:]))
    assert errs[-1] < 1e-15


def test_ozaki_kchunk_matches_within_rounding():
    A = uniform(14, (20, 130), np.float64)
    B = uniform(15, (130, 21), np.float64)
    a = oracle.ozaki_gemm(A, B, 7, kchunk=0)
    b = oracle.ozaki_gemm(A, B, 7, kchunk=32)
    np.testing.assert_allclose(a, b, rtol=1e-14, atol=1e-15)


def test_ozaki_alpha_beta():
    A = uniform(16, (10, 30), np.float64)
    B = uniform(17, (30, 9), np.float64)
    Cin = uniform(18, (10, 9), np.float64)
    out = oracle.ozaki_gemm(A, B, 9, Cin=Cin, alpha=2.0, beta=0.5)
    np.testing.assert_allclose(out, 2.0 * (A @ B) + 0.5 * Cin, rtol=1e-13, atol=1e-14)


def _packed_slice_words(row, e, s):
    """Python statement of the device's packed slicing (split_device.cuh,
    fixed_of / digit_at / slice4_packed): per 4 consecutive values, the
    fixed-point F = floor(|v| 2^(7s - e)) from the FP64 bits, digit t of
    value j shifted into byte j of word t, the negative values' bytes negated
    as (0x80808080 - w) ^ 0x80808080, and the magnitude sum F >> (7s - 30)."""
    import struct

    m32 = 0xFFFFFFFF
    words, mags = [], []
    for c in range(0, len(row), 4):
        lo, hi, nm, mag = [], [], 0, 0
        for j, v in enumerate(row[c:c + 4]):
            bits = struct.unpack("<Q", struct.pack("<d", float(v)))[0]
            ex, mant = (bits >> 52) & 0x7FF, bits & ((1 << 52) - 1)
            sig = (mant | (1 << 52)) if ex else mant
            sh = 7 * s - e + (ex if ex else 1) - 1075
            f = (0 if sh >= 64 else (sig << sh) & ((1 << 64) - 1)) if sh >= 0 else (0 if -sh >= 64 else sig >> -sh)
            lo.append(f & m32)
            hi.append(f >> 32)
            if bits >> 63:
                nm |= 0xFF << (8 * j)
            mag += f >> (7 * s - 30) if 7 * s >= 30 else 0
        row_words = []
        for t in range(s):
            o, x = 7 * (s - 1 - t), 0
            for j in range(4):
                n = o - 8 * j
                y = hi[j] >> (n - 32) if n >= 32 else (((hi[j] << 32 | lo[j]) >> n) & m32 if n > 0 else (lo[j] << -n) & m32)
                x |= y & (127 << (8 * j))
            nx = ((0x80808080 - x) & m32) ^ 0x80808080
            row_words.append((x & ~nm & m32) | (nx & nm))
        words.append(row_words)
        mags.append(mag)
    return words, mags


@pytest.mark.parametrize("s", [4, 5, 6, 7, 8, 9])
def test_packed_slice_words_match_the_slicing(s):
    """The word-at-a-time slicing of the device pre-passes gives, byte for
    byte, the restatement's slices (the FP64 truncation sequence), and its
    magnitude sums equal ozaki_magnitude_sums: rows with wide exponent
    ranges, negative and signed-zero entries, subnormals and a zero row."""
    rng = np.random.default_rng(40 + s)
    m, k = 12, 32
    A = rng.uniform(-1, 1, (m, k)) * 10.0 ** rng.integers(-30, 30, (m, k))
    A[1, ::3] = -0.0
    A[2] = 0.0
    A[3] = rng.uniform(-1, 1, k) * 1e-310  # subnormal row
    A[4, 5] = 1e300
    B = np.ones((k, 1))
    ea, _, sa, _ = oracle.ozaki_slices(A, B, s)
    rows_sums, _ = oracle.ozaki_magnitude_sums(A, B)
    for r in range(m):
        words, mags = _packed_slice_words(A[r], int(ea[r]), s)
        for g, row_words in enumerate(words):
            for t, w in enumerate(row_words):
                expect = bytes(sa[t, r, 4 * g:4 * g + 4].view(np.uint8))
                assert w.to_bytes(4, "little") == expect, (r, g, t)
        if 7 * s >= 30:
            assert sum(mags) == rows_sums[r]
