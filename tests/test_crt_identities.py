"""The integer identities the CRT kernels rest on, checked exactly on the CPU (Python integers
and rationals; no GPU).

* reconstruction: moduli in pairs share the factor Q_g = P / (p_2g p_2g+1) of their CRT weights,
  W_l = Q_g X_l with X_l < 2^16, so sum_l r_l W_l = sum_g Q_g (r_2g X_2g + r_2g+1 X_2g+1)
  exactly, each pair sum < 2^25 and each 32-bit limb column < 2^60;
* split: for |t| <= 2^62 = hi 2^32 + lo, one FMA s = hi (2^32 mod p) + lo (exact, < 2^39) and
  one FMA with 1.5 2^52 give q = rint(s / p), and lo + hi c32 - q p (mod 2^32) is the symmetric
  residue of t for every odd modulus; for p = 256 it is t's low byte;
* GEMM epilogue: v + bias with bias = p ceil((2^31 - 2^21) / p) lies in [0, 2^32) for every
  accumulator |v| <= 1023 * 128^3 and reduces to v mod p with one unsigned Barrett step.
"""
from __future__ import annotations

import random
import struct
from fractions import Fraction

import pytest

# the moduli of crt_modulus() (eigen_b200/csrc/kernels.h): pairwise coprime, 256 first
MODULI = [256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193, 191, 181, 179, 173]


def crt_weights(n):
    P = 1
    for p in MODULI[:n]:
        P *= p
    W = [(P // p) * pow(P // p, -1, p) for p in MODULI[:n]]
    return P, W


def pair_table(n):
    P, _ = crt_weights(n)
    X, Q = [0] * n, []
    for g in range(0, n, 2):
        pa = MODULI[g]
        pb = MODULI[g + 1] if g + 1 < n else 1
        Q.append(P // (pa * pb))
        X[g] = pb * pow(P // pa, -1, pa)
        if g + 1 < n:
            X[g + 1] = pa * pow(P // pb, -1, pb)
    return P, X, Q


@pytest.mark.parametrize("n", range(1, 17))
def test_pair_weights_reproduce_the_crt_weights(n):
    P, W = crt_weights(n)
    _, X, Q = pair_table(n)
    assert P < 2**128
    for l in range(n):
        assert Q[l // 2] * X[l] == W[l]
        assert X[l] < 2**16
    rng = random.Random(n)
    for _ in range(200):
        r = [rng.randrange(p) for p in MODULI[:n]]
        s_direct = sum(ri * wi for ri, wi in zip(r, W))
        sums = [r[g] * X[g] + (r[g + 1] * X[g + 1] if g + 1 < n else 0) for g in range(0, n, 2)]
        assert all(s < 2**25 for s in sums)
        assert sum(Q[g] * R for g, R in enumerate(sums)) == s_direct
        # the four 32-bit limb columns of sum_g Q_g R_g stay below 2^60
        for q in range(4):
            col = sum(((Q[g] >> (32 * q)) & 0xFFFFFFFF) * R for g, R in enumerate(sums))
            assert col < 2**60
        # and the value reconstructs: S mod P is the number the residues encode
        x = s_direct % P
        assert all(x % p == ri for p, ri in zip(MODULI[:n], r))


def _rn(x: Fraction) -> float:
    """x rounded to the nearest double (ties to even): Python's float(Fraction) is correctly rounded."""
    return float(x)


def _fma(a: float, b: float, c: float) -> float:
    return _rn(Fraction(a) * Fraction(b) + Fraction(c))


def _low_word(d: float) -> int:
    return struct.unpack("<Q", struct.pack("<d", d))[0] & 0xFFFFFFFF


def split_residue(t: int, p: int) -> int:
    """The split kernel's residue of t for modulus p, as an int8 value."""
    hi, lo = t >> 32, t & 0xFFFFFFFF
    if p == 256:
        r = lo & 0xFF
    else:
        c32 = (1 << 32) % p
        s = _fma(float(hi), float(c32), float(lo))
        q = _low_word(_fma(s, 1.0 / p, 1.5 * 2.0**52))
        r = (lo + (hi & 0xFFFFFFFF) * c32 - q * p) & 0xFFFFFFFF
        r &= 0xFF
    return r - 256 if r >= 128 else r


def test_split_residue_is_the_symmetric_residue():
    rng = random.Random(3)
    ts = [0, 1, -1, 2**62, -(2**62), 2**62 - 1, -(2**62) + 1, 2**32, -(2**32), 2**31 - 1]
    ts += [rng.randrange(-(2**62), 2**62 + 1) for _ in range(300)]
    ts += [rng.randrange(-(2**40), 2**40) for _ in range(100)]
    for t in ts:
        for p in MODULI[:16]:
            got = split_residue(t, p)
            m = t % p
            want = m - p if m > (p - 1) // 2 else m  # symmetric: [-(p-1)/2, (p-1)/2], p = 256: [-128, 127]
            if p == 256:
                want = m - 256 if m >= 128 else m
            assert got == want, (t, p, got, want)


def test_epilogue_bias_reduction():
    lim = 1023 * 128 * 128 * 128
    assert lim == 2**31 - 2**21
    rng = random.Random(5)
    for p in MODULI:
        magic = (2**32 - 1) // p
        bias = (0x7FE00000 + p - 1) // p * p
        assert bias % p == 0 and lim <= bias < lim + p
        for v in [-lim, lim, 0, -1, 1] + [rng.randint(-lim, lim) for _ in range(400)]:
            u = v + bias
            assert 0 <= u < 2**32
            r = u - ((u * magic) >> 32) * p
            if r >= p:
                r -= p
            assert r == v % p
