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
