"""The argument behind the CRT reconstruction's one-rounding fast paths (CPU).

`crt_round` in eigen_b200/csrc/crt.cu rounds the exact remainder R (|R| < P/2, 128-bit two's
complement) to the nearest double of R 2^escale without the magnitude path in the common case:

* hi = the signed 64-bit window of R at limbs kW, kW+1, lo = the limbs below it;
* |hi| >= 2^54: RN(hi | [lo != 0]) 2^(32 kW);
* 8 <= |hi| < 2^54: R = h 2^(32 kW + 1) + X, h = hi >> 1; kW = 1: RN(h 2^33 + X); kW = 2:
  RN(h 2^53 + ((X >> 12) | [X mod 2^12 != 0])) 2^12;
* the result is kept when it stays normal after scaling.

This test restates those steps with exact Python integers (int -> float conversion rounds to
nearest even, like the device conversions and the FMA of exact operands) and checks them
against the exactly rounded value of R 2^escale on random remainders, exact ties, lone sticky
bits and the window thresholds, for 16 (kW = 2) and 11 (kW = 1) moduli.  The device code
itself is checked bit for bit against the oracle by tests/test_crt_gpu.py.
"""
from __future__ import annotations

import math
import random
from fractions import Fraction

import pytest

from _helpers import crt_model

DBL_MIN = 2.0 ** -1022


def exact_rn(R: int, escale: int) -> float:
    """Nearest double (ties to even) of R 2^escale, for results in the normal range."""
    x = Fraction(R) * Fraction(2) ** escale
    if x == 0:
        return 0.0
    sign = -1.0 if x < 0 else 1.0
    x = abs(x)
    e = math.floor(math.log2(x.numerator) - math.log2(x.denominator))
    while Fraction(2) ** e > x:
        e -= 1
    while Fraction(2) ** (e + 1) <= x:
        e += 1
    ulp = Fraction(2) ** (e - 52)
    q, r = divmod(x, ulp)
    if r * 2 > ulp or (r * 2 == ulp and q % 2 == 1):
        q += 1
    return sign * math.ldexp(float(q), e - 52)


def fast_path(R: int, escale: int, kw: int):
    """The fast paths of crt_round as stated above; None where the device takes the magnitude
    path (|hi| < 8 or a result outside the normal range)."""
    mask = (1 << (32 * kw)) - 1
    hi = R >> (32 * kw)  # floor: the signed window
    lo = R & mask
    if -8 <= hi < 8:
        return None
    if hi >= 1 << 54 or hi < -(1 << 54):
        d = float(hi | (1 if lo else 0))
        s = 32 * kw
    elif kw == 1:
        h = hi >> 1
        X = ((hi & 1) << 32) | lo
        d = float(h * 2 ** 33 + X)  # one rounding of exact operands, as the FMA
        s = 0
    else:
        h = hi >> 1
        X = ((hi & 1) << 64) | lo
        x = (X >> 12) | (1 if X & 0xFFF else 0)
        assert x < 1 << 53
        d = float(h * 2 ** 53 + x)
        s = 12
    try:
        v = math.ldexp(d, s + escale)
    except OverflowError:  # the device adds to the exponent only while the result stays normal
        return None
    if v == 0.0 or abs(v) < DBL_MIN or math.isinf(v):
        return None
    return v


def remainders(bits: int, rng: random.Random, count: int):
    """Random |R| < 2^bits, exact ties and lone sticky bits at random positions, values around
    the window thresholds, both signs."""
    for _ in range(count):
        kind = rng.randrange(6)
        L = rng.randrange(1, bits + 1)
        if kind == 0:
            m = rng.getrandbits(L)
        elif kind == 1:  # a tie: bits below the 53-bit window are exactly 100..0
            top = rng.getrandbits(53) | (1 << 52)
            sh = rng.randrange(1, max(2, L - 53))
            m = (top << sh) | (1 << (sh - 1))
        elif kind == 2:  # just above a tie: a lone sticky bit far below
            top = rng.getrandbits(53) | (1 << 52)
            sh = rng.randrange(2, max(3, L - 53))
            m = (top << sh) | (1 << (sh - 1)) | (1 << rng.randrange(0, sh - 1))
        elif kind == 3:  # at the |hi| = 2^54 threshold of the 64-bit window
            base = 1 << (54 + 32 * (2 if bits > 96 else 1))
            m = base + rng.randrange(-(1 << 40), 1 << 40)
        elif kind == 4:  # at the |hi| = 8 threshold
            base = 8 << (32 * (2 if bits > 96 else 1))
            m = base + rng.randrange(-(1 << 33), 1 << 33)
        else:  # exactly representable values and their neighbours
            m = (rng.getrandbits(53) | (1 << 52)) << rng.randrange(0, max(1, L - 53))
            m += rng.choice([-1, 0, 1])
        m = min(max(m, 0), (1 << bits) - 1)
        yield -m if rng.random() < 0.5 else m


@pytest.mark.parametrize("moduli,kw", [(16, 2), (11, 1)])
def test_fast_paths_round_like_exact_rounding(moduli, kw):
    P = crt_model().modulus_product(moduli)
    bits = (P // 2).bit_length()
    assert (P // 2) < 1 << (63 + 32 * kw)  # the window holds every R in [-P/2, P/2)
    rng = random.Random(moduli)
    seen = {"conversion": 0, "fma": 0, "tie": 0}
    for R in remainders(bits, rng, 60000):
        if R >= P // 2 or R < -(P // 2):
            continue
        escale = rng.choice([0, -60, -120, -900, -1000 - rng.randrange(80), 800 + rng.randrange(150),
                             rng.randrange(-1100, 1000)])
        got = fast_path(R, escale, kw)
        if got is None:
            continue
        assert got == exact_rn(R, escale), (R, escale)
        hi = R >> (32 * kw)
        seen["conversion" if (hi >= 1 << 54 or hi < -(1 << 54)) else "fma"] += 1
        L = abs(R).bit_length()
        seen["tie"] += L > 54 and abs(R) & ((1 << (L - 53)) - 1) == 1 << (L - 54)
    assert seen["conversion"] > 2000 and seen["fma"] > 2000 and seen["tie"] > 1000, seen
