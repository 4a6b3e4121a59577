"""The integer-slice arithmetic of the tensor-core far field (csrc/hmat_tc.cu), restated in
numpy on the CPU: operands cut into six signed 7-bit slices of 42-bit fixed-point values
(exponent with one bit of headroom), the 21 slice pairs with t + u <= 5 (0-based) summed per
group g = t + u in exact integers, and the FP64 epilogue sum_g 2^-7(g+2) A_g scaled by
2^(e_r + f_n).

* the slices reproduce each operand to 2^-41 of its row / state maximum;
* a tile row's dot product over K = 2048 matches the exact (rational) value to 1e-12 of
  sum |a_k b_k|, for FP32 factors and FP64 states, with and without cancellation;
* every group sum stays inside int32 at the largest tile (K = 2048 in the plan; 8192 is the
  cap of SPX_TC_KSTEP x 32).
"""
from fractions import Fraction

import numpy as np

FIX, NSL, NG = 42, 6, 6


def headroom_exp(mx):
    return int(np.floor(np.log2(mx))) + 2 if mx > 0 else 0


def slices6(v, e):
    """int slices d[0..5] of v (|v| < 2^(e-1)), most significant first."""
    m = int(np.rint(np.ldexp(float(v), FIX - e)))
    a = abs(m)
    q = [(a >> (FIX - 7 * (t + 1))) & 127 for t in range(NSL)]
    return [-x if m < 0 else x for x in q]


def tile_dot(a, b):
    """The kernel's value of sum_k a_k b_k for one tile row and one state."""
    er = headroom_exp(np.abs(a).max())
    fn = headroom_exp(np.abs(b).max())
    da = np.array([slices6(x, er) for x in a], dtype=np.int64)   # [K][6]
    cb = np.array([slices6(x, fn) for x in b], dtype=np.int64)
    groups = np.zeros(NG, dtype=np.int64)
    for t in range(NSL):
        for u in range(NG - t):
            groups[t + u] += int(np.dot(da[:, t], cb[:, u]))
    y = 0.0
    for g in range(NG - 1, -1, -1):
        y += np.ldexp(float(groups[g]), -7 * (g + 2))
    return np.ldexp(y, er + fn), groups


def exact_dot(a, b):
    return float(sum(Fraction(float(x)) * Fraction(float(y)) for x, y in zip(a, b)))


def test_slices_reproduce_operands():
    rng = np.random.default_rng(1)
    v = rng.standard_normal(64) * 10.0 ** rng.uniform(-3, 3, 64)
    e = headroom_exp(np.abs(v).max())
    for x in v:
        d = slices6(x, e)
        assert all(-127 <= q <= 127 for q in d)
        back = sum(q * 2.0 ** (-7 * (t + 1)) for t, q in enumerate(d)) * 2.0 ** e
        assert abs(back - x) <= 2.0 ** (e - FIX)


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
        y, groups = tile_dot(a.astype(np.float64), b)
        ex = exact_dot(a, b)
        scale = float(np.sum(np.abs(a.astype(np.float64) * b)))
        assert abs(y - ex) <= 1e-12 * scale, (case, y, ex, scale)
        assert np.abs(groups).max() < 2 ** 31


def test_group_sums_fit_int32_at_the_cap():
    # the extreme: every slice at +-127, six pairs in one group, K = 8192
    assert 6 * 8192 * 127 * 127 < 2 ** 31
