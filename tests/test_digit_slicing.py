"""The arithmetic of the exact tensor-core stages (csrc/vg_oz.cu), restated on
the host and checked exactly with rational arithmetic:

- to_digits16: t = fma(v, 2^(38 - E), 2^52 + 0x8080808080) holds
  u = rint(v 2^(38 - E)) + 0x8080808080 in its low 40 mantissa bits, and the
  five bytes of u less 128 are balanced digits (-128 .. 127) whose
  base-256 value is the fixed-point integer xi, |xi| < 2^38, for every value
  of a scale group whose maximum is below 2^E;
- the level sums: for contractions of 32, 96 and 512 terms (with every value
  at its group's maximum for the longest) every level accumulator stays
  inside int32 (a level holds at most 5 K 2^14, below 2^31 for K under
  26 000), and keeping
  levels 0 .. 4 (15 digit-pair products) leaves an error below
  K 2^-36 |x|max |y|max per dot product against the exact product of the
  fixed-point operands;
- combine_levels: the five levels summed in 64-bit integers (within the
  levels' bounds the sum stays below 2^56) and converted as hi 2^32 + lo with
  one FMA equal the correctly rounded value of the kept sum times the
  power-of-two scale.
"""
import math
import random
from fractions import Fraction

import numpy as np

FIX_BITS = 38
MAGIC = Fraction(2 ** 52 + 0x8080808080)


def rn(q):
    """q (a Fraction) rounded to the nearest double, ties to even."""
    return float(q)


def digits(v, E):
    """to_digits16 for one value: (xi, five digits, most significant first)."""
    t = rn(Fraction(v) * Fraction(2) ** (FIX_BITS - E) + MAGIC)
    m = Fraction(t) - 2 ** 52  # t lies in [2^52, 2^53): its low mantissa bits are exact
    assert m.denominator == 1
    u = int(m)
    assert 0 <= u < 2 ** 40
    d = [((u >> (8 * (4 - s))) & 0xFF) - 128 for s in range(5)]
    xi = u - 0x8080808080
    return xi, d


def group_exp(mx):
    return math.frexp(mx)[1] if mx > 0 else 0


def sample_group(rng, n):
    """n values of one scale group: mixed magnitudes, signs, exact zeros."""
    top = 10.0 ** rng.uniform(-30, 30)
    out = []
    for _ in range(n):
        r = rng.random()
        if r < 0.05:
            out.append(0.0)
        elif r < 0.1:
            out.append(top * (1 if rng.random() < 0.5 else -1))
        else:
            out.append(top * rng.uniform(-1, 1) * 10.0 ** rng.uniform(-12, 0))
    return out


def test_digits_reconstruct_the_fixed_point_value():
    rng = random.Random(7)
    for _ in range(200):
        vals = sample_group(rng, 16)
        E = group_exp(max(abs(v) for v in vals))
        for v in vals:
            xi, d = digits(v, E)
            assert all(-128 <= x <= 127 for x in d)
            assert sum(x * 256 ** (4 - s) for s, x in enumerate(d)) == xi
            assert abs(xi) < 2 ** FIX_BITS
            # xi is v 2^(38-E) rounded to the nearest integer (ties to even)
            exact = Fraction(v) * Fraction(2) ** (FIX_BITS - E)
            assert abs(exact - xi) <= Fraction(1, 2)


def test_levels_fit_int32_and_bound_the_dropped_terms():
    rng = random.Random(11)
    for K in (32, 96, 512):
        for _ in range(3):
            x = sample_group(rng, K)
            y = sample_group(rng, K)
            # worst case for the accumulators: every value at the group maximum
            if K == 512:
                x = [max(abs(v) for v in x)] * K
                y = [-max(abs(v) for v in y)] * K
            Ex, Ey = group_exp(max(abs(v) for v in x)), group_exp(max(abs(v) for v in y))
            dx = [digits(v, Ex) for v in x]
            dy = [digits(v, Ey) for v in y]
            acc = [0] * 9
            for (xi, a), (yi, b) in zip(dx, dy):
                for s in range(5):
                    for t in range(5):
                        acc[s + t] += a[s] * b[t]
            for lam in range(5):
                assert -(2 ** 31) <= acc[lam] < 2 ** 31
            exact = sum(xi * yi for (xi, _), (yi, _) in zip(dx, dy))
            kept = sum(acc[lam] * 2 ** (64 - 8 * lam) for lam in range(5))
            assert abs(exact - kept) < K * 2 ** (2 * FIX_BITS - 36)


def combine(a, sc):
    """combine_levels: the 64-bit sum, split hi / lo, one FMA (emulated exactly)."""
    t = (a[0] << 32) + (a[1] << 24) + (a[2] << 16) + (a[3] << 8) + a[4]
    assert -(2 ** 63) <= t < 2 ** 63  # the level bounds keep |t| below 2^56
    hi, lo = t >> 32, t & 0xFFFFFFFF
    assert float(hi) == hi and float(lo) == lo
    return rn(Fraction(hi) * Fraction(sc) * 2 ** 32 + Fraction(lo) * Fraction(sc)), t


def test_combine_levels_rounds_once():
    rng = np.random.default_rng(3)
    for _ in range(2000):
        # level lam holds at most (lam + 1) digit pairs of |d g| <= 2^14 per K step, K <= 512
        a = [int(rng.integers(-(lam + 1) * 512 * 2 ** 14, (lam + 1) * 512 * 2 ** 14 + 1)) for lam in range(5)]
        sc = 2.0 ** int(rng.integers(-200, 100))
        got, t = combine(a, sc)
        assert got == rn(Fraction(t) * Fraction(sc))
        assert t == sum(a[lam] * 2 ** (32 - 8 * lam) for lam in range(5))
