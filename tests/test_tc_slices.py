"""The integer-digit arithmetic of the tensor-core far field (csrc/hmat_tc.cu), restated in
numpy on the CPU: an operand is the fixed-point integer llrint(v 2^(8 nd - 1 - e)) (e with one
bit of headroom over the largest |v| of the tile row / state range) cut into nd balanced
base-256 digits in [-128, 127] (nd = 4 for the FP32 factors, 6 for the FP64 states); all 24
digit pairs are summed in exact integers (D_tu = sum_k d_tk c_uk, what one kind::i8 MMA of
N = 48 accumulates per A digit t), and the FP64 epilogue is sum_{t,u} 256^(8 - t - u) D_tu
scaled by 2^(e_r + f_n - 78).

* the digits reproduce each operand's fixed-point value exactly, so an operand is exact to
  2^(e - 8 nd) (FP32 factors within 2^7 of their row maximum are exact);
* a tile row's dot product over K = 2048 matches the exact (rational) value within the
  rounding bound of the two fixed points (half a unit of the last digit of each operand) and
  to 1e-10 of sum |a_k b_k|, for FP32 factors and FP64 states, with and without cancellation.
  The FP32 rounding of the factors themselves (2^-24 relative per element) weighs about 100x
  more than this;
* every pair sum stays inside int32 at the largest tile (K = 2048 in the plan; 8192 is the
  cap of SPX_TC_KSTEP x 32).
"""
from fractions import Fraction

import numpy as np

NDA, NDB = 4, 6


def headroom_exp(mx):
    return int(np.floor(np.log2(mx))) + 2 if mx > 0 else 0


def digits(v, e, nd):
    """balanced base-256 digits d[0..nd-1] of llrint(v 2^(8 nd - 1 - e)), most significant first."""
    m = int(np.rint(np.ldexp(float(v), 8 * nd - 1 - e)))
    d = [0] * nd
    for t in range(nd - 1, -1, -1):
        lo = m & 255
        s = lo - 256 if lo >= 128 else lo
        d[t] = s
        m = (m - s) >> 8
    assert m == 0
    return d


def tile_dot(a, b):
    """The kernel's value of sum_k a_k b_k for one tile row and one state."""
    er = headroom_exp(np.abs(a).max())
    fn = headroom_exp(np.abs(b).max())
    da = np.array([digits(x, er, NDA) for x in a], dtype=np.int64)   # [K][4]
    cb = np.array([digits(x, fn, NDB) for x in b], dtype=np.int64)   # [K][6]
    D = da.T @ cb                                                    # [t][u], exact
    y = 0.0
    for t in range(NDA):
        for u in range(NDB):
            y += float(D[t, u]) * 2.0 ** (8 * (8 - t - u))
    return np.ldexp(y, er + fn - (8 * NDA - 1) - (8 * NDB - 1)), D


def exact_dot(a, b):
    return float(sum(Fraction(float(x)) * Fraction(float(y)) for x, y in zip(a, b)))


def test_digits_reproduce_operands():
    rng = np.random.default_rng(1)
    v = rng.standard_normal(64) * 10.0 ** rng.uniform(-3, 3, 64)
    e = headroom_exp(np.abs(v).max())
    for nd in (NDA, NDB):
        fix = 8 * nd - 1
        for x in v:
            d = digits(x, e, nd)
            assert all(-128 <= q <= 127 for q in d)
            m = sum(q * 256 ** (nd - 1 - t) for t, q in enumerate(d))
            assert m == int(np.rint(np.ldexp(x, fix - e)))
            assert abs(np.ldexp(float(m), e - fix) - x) <= 2.0 ** (e - fix - 1)
    # FP32 values within 2^7 of the maximum are exact
    f = (rng.standard_normal(256)).astype(np.float32)
    e = headroom_exp(float(np.abs(f).max()))
    for x in f:
        if abs(float(x)) >= 2.0 ** (e - 8):
            m = sum(q * 256 ** (3 - t) for t, q in enumerate(digits(float(x), e, NDA)))
            assert np.ldexp(float(m), e - (8 * NDA - 1)) == float(x)


def test_tile_dot_matches_exact_value():
    rng = np.random.default_rng(2)
    K = 2048
    for case in range(3):
        a = (rng.standard_normal(K) / np.sqrt(K)).astype(np.float32)
        if case == 0:
            b = rng.standard_normal(K)                                   # random states
        elif case == 1:
            b = 1.0 + 0.01 * np.cos(np.linspace(0, 6.0, K))              # smooth, large mean
        else:
            b = np.cos(np.linspace(0, 60.0, K)) * 1e-3 + 5.0              # cancellation
            a = (a - a.mean()).astype(np.float32)
        y, D = tile_dot(a.astype(np.float64), b)
        ex = exact_dot(a, b)
        a64 = a.astype(np.float64)
        scale = float(np.sum(np.abs(a64 * b)))
        # rounding of the two fixed points: half a unit of each operand's last digit
        er, fn = headroom_exp(np.abs(a64).max()), headroom_exp(np.abs(b).max())
        bound = float(np.sum(np.abs(b)) * 2.0 ** (er - 8 * NDA) + np.sum(np.abs(a64)) * 2.0 ** (fn - 8 * NDB))
        assert abs(y - ex) <= bound + 1e-15 * scale, (case, y, ex, bound)
        assert abs(y - ex) <= 1e-10 * scale, (case, y, ex, scale)
        assert np.abs(D).max() < 2 ** 31


def test_pair_sums_fit_int32_at_the_cap():
    # the extreme: every digit at -128, K = 8192 (one pair per accumulator column)
    assert 8192 * 128 * 128 < 2 ** 31


def digits6_split(v, e):
    """The kernel's 32-bit form of digits(v, e, 6): m = hi 2^24 + lo, three balanced digits of
    lo, the carry into hi, three digits of hi."""
    m = int(np.rint(np.ldexp(float(v), 8 * NDB - 1 - e)))
    lo, hi = m & 0xFFFFFF, m >> 24
    d = [0] * 6
    for t in (5, 4, 3):
        q = ((lo & 255) ^ 128) - 128
        d[t] = q
        lo = (lo - q) >> 8
    assert lo in (0, 1)
    hi += lo
    for t in (2, 1):
        q = ((hi & 255) ^ 128) - 128
        d[t] = q
        hi = (hi - q) >> 8
    d[0] = hi
    return d


def test_split_digits_equal_the_generic_ones():
    rng = np.random.default_rng(3)
    v = np.concatenate([rng.standard_normal(2000) * 10.0 ** rng.uniform(-6, 0, 2000), [0.0, 1.0, -1.0]])
    e = headroom_exp(np.abs(v).max())
    for x in v:
        d = digits6_split(x, e)
        assert d == digits(x, e, NDB)
        assert all(-128 <= q <= 127 for q in d)
    # the extremes of the 47-bit range
    for m in (2 ** 46, -2 ** 46, 2 ** 46 - 1, -(2 ** 46 - 1), 2 ** 24 - 1, -(2 ** 24)):
        x = np.ldexp(float(m), 1 - (8 * NDB - 1))  # e = 1
        assert digits6_split(x, 1) == digits(x, 1, NDB)
