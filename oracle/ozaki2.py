"""Exact CPU model of the CRT-form (Ozaki scheme II) emulated FP64 product.

Test infrastructure only: the GPU path (the CRT mode of the tcgen05 slice GEMM and the
residue split / reconstruction kernels) must reproduce these results bit for bit.  The
model does not use residues at all: since |C'_ij| < P/2, the CRT reconstruction of the
device equals the exact integer product C' = A' B'^T, which Python integers give
directly.  What the model does restate exactly is every floating-point step that decides
the result:

  * e_r: exponent of the row maximum (max |x| in [2^(e-1), 2^e));
  * per 128-column chunk c: S_c = sum over nonzero x of ceil(rn(x'^2) 2^32) + 1, with
    x' = x 2^-e_c (e_c: exponent of the chunk maximum) computed as two exact power-of-two
    products (``scale2``); folded into S_r = sum_c ceil(S_c 4^(e_c - e)), an integer upper
    bound of ||x||^2 2^(32-2e);
  * mu_r = b - (e - 16 + ceil(L/2)), L = bit length of S_r - 1 (0 for a zero row);
  * A'_rl = trunc(scale2(x_rl, mu_r)) as an exact integer;
  * C_ij = alpha * RN(RN(C'_ij) 2^-(mu_i + nu_j))  [+ beta C_ij as one fused multiply-add].

Reference semantics: C = alpha op(A) op(B) + beta C of Eigen's BLAS dgemm_
(blas/level3_impl.h:61-96 in the Eigen tree), here with the emulated product in place of
Eigen's gebp kernel.  Sizes are meant for tests (Python integer arithmetic).
"""
from __future__ import annotations

import math
from fractions import Fraction

import numpy as np

MODULI = [256, 255, 253, 251, 247, 241, 239, 233, 229, 227,
          223, 217, 211, 199, 197, 193, 191, 181, 179, 173]


def modulus_product(n: int) -> int:
    P = 1
    for p in MODULI[:n]:
        P *= p
    return P


def bits(n: int) -> int:
    """Largest b with 2^(2b+1) < P (so |C'| <= 2^(2b) < P/2)."""
    P = modulus_product(n)
    b = (P.bit_length() - 2) // 2
    while 2 ** (2 * b + 1) >= P:
        b -= 1
    return b


def _c_div(a: int, b: int) -> int:
    """C integer division (truncation toward zero)."""
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b >= 0) else -q


def scale2(x: float, e: int) -> float:
    """x * 2^e as two power-of-two products, each rounded to nearest (float64)."""
    e1 = _c_div(e, 2)
    return float(np.float64(np.float64(x) * np.float64(math.ldexp(1.0, e1))) * np.float64(math.ldexp(1.0, e - e1)))


CHUNK = 128  # columns (along K) per norm-bound chunk


def row_mu(row: np.ndarray, b: int) -> int:
    """Scale exponent of one row from chunked integer norm bounds: per 128-column chunk c,
    S_c = sum over nonzero x of ceil(rn(x'^2) 2^32) + 1 with x' = x 2^-e_c (e_c: exponent of
    the chunk maximum); S = sum_c ceil(S_c 4^(e_c - e)) with e the row maximum's exponent;
    mu = b - (e - 16 + ceil(L/2)), L the bit length of S - 1."""
    row = np.asarray(row, dtype=np.float64)
    mx = float(np.max(np.abs(row))) if row.size else 0.0
    if mx == 0.0 or not math.isfinite(mx):
        return 0
    e = math.frexp(mx)[1]
    S = 0
    for c0 in range(0, row.size, CHUNK):
        chunk = row[c0:c0 + CHUNK]
        cmx = float(np.max(np.abs(chunk)))
        if cmx == 0.0:
            continue
        ec = math.frexp(cmx)[1]
        Sc = 0
        for x in chunk:
            x = float(x)
            if x != 0.0:
                xs = scale2(x, -ec)
                sq = float(np.float64(xs) * np.float64(xs))
                Sc += int(math.ceil(sq * 4294967296.0)) + 1
        sh = 2 * (e - ec)
        S += 1 if sh >= 64 else ((Sc - 1) >> sh) + 1
    L = (S - 1).bit_length() if S > 1 else 0
    return b - (e - 16 + (L + 1) // 2)


def scaled_integers(X: np.ndarray, b: int):
    """(mu, X') with X'_rl = trunc(x_rl 2^mu_r) as Python integers (object array)."""
    X = np.asarray(X, dtype=np.float64)
    rows, cols = X.shape
    mu = [row_mu(X[r], b) for r in range(rows)]
    Xi = np.empty((rows, cols), dtype=object)
    for r in range(rows):
        for l in range(cols):
            Xi[r, l] = int(math.trunc(scale2(float(X[r, l]), mu[r])))
    return mu, Xi


def _ldexp_rn(d: float, e: int) -> float:
    try:
        return math.ldexp(d, e)
    except OverflowError:
        return math.copysign(math.inf, d)


def _fma(a: float, b: float, c: float) -> float:
    r = Fraction(a) * Fraction(b) + Fraction(c)
    try:
        return float(r)
    except OverflowError:
        return math.copysign(math.inf, float(r.numerator))


def crt_dgemm(opA: np.ndarray, opB: np.ndarray, alpha: float, beta: float, C: np.ndarray, moduli: int = 16):
    """C <- alpha opA opB + beta C through the CRT emulation model (opA: m x k, opB: k x n).

    Returns (C_new, info) with info = {"b", "mu", "nu", "max_abs_cprime"}."""
    opA = np.asarray(opA, dtype=np.float64)
    opB = np.asarray(opB, dtype=np.float64)
    m, k = opA.shape
    n = opB.shape[1]
    b = bits(moduli)
    P = modulus_product(moduli)
    mu, Ai = scaled_integers(opA, b)
    nu, Bi = scaled_integers(opB.T, b)
    Cp = Ai.dot(Bi.T) if k else np.zeros((m, n), dtype=object)
    out = np.array(C, dtype=np.float64, copy=True)
    big = 0
    for i in range(m):
        for j in range(n):
            c = int(Cp[i, j])
            big = max(big, abs(c))
            assert 2 * abs(c) < P, "C' outside the CRT range"
            val = _ldexp_rn(float(c), -(mu[i] + nu[j])) if c else 0.0
            v = float(np.float64(alpha) * np.float64(val))
            out[i, j] = v if beta == 0.0 else _fma(beta, float(out[i, j]), v)
    return out, {"b": b, "mu": mu, "nu": nu, "max_abs_cprime": big}
