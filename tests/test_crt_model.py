"""The CRT-form emulation model (oracle/ozaki2.py) on the CPU: its constants, its
accuracy against the double-double oracle, and the residue route the GPU takes
(residues, products mod p, Chinese-remainder reconstruction) against its exact product."""
from __future__ import annotations

import math

import numpy as np

from _helpers import U64, crt_model, dd_reference, make_operands, op, rel_error_vs_dd


def test_moduli_pairwise_coprime_and_bits():
    M = crt_model()
    mods = M.MODULI
    assert len(mods) == 20 and all(p <= 256 for p in mods)
    for i in range(len(mods)):
        for j in range(i):
            assert math.gcd(mods[i], mods[j]) == 1
    assert M.bits(16) == 62 and M.bits(18) == 69 and M.bits(20) == 77
    for n in range(8, 21):
        b = M.bits(n)
        P = M.modulus_product(n)
        assert 2 ** (2 * b + 1) < P <= 2 ** (2 * b + 3)


def test_row_scaling_bounds_the_norm():
    """||trunc(2^mu x)||_2 <= 2^b, and the bound is within a factor 2 of tight."""
    M = crt_model()
    rng = np.random.default_rng(1)
    for r in (0, 10, 200):
        X = rng.uniform(-1, 1, (20, 300)) * 2.0 ** rng.integers(-r, r + 1, (20, 300))
        X[3] = 0.0
        mu, Xi = M.scaled_integers(X, 62)
        for i in range(20):
            nrm2 = sum(int(v) * int(v) for v in Xi[i])
            if i == 3:
                assert nrm2 == 0
                continue
            assert nrm2 <= 2 ** 124
            exact = math.fsum(float(x) ** 2 for x in X[i]) * 4.0 ** mu[i]
            assert exact > 2.0 ** 120  # 2^mu ||x|| > 2^(b-2)


def test_model_accuracy_vs_double_double():
    M = crt_model()
    for r in (0, 16):
        m, n, k = 48, 40, 300
        A, lda, B, ldb, C, ldc = make_operands(m, n, k, r=r, seed=r + 3)
        out, info = M.crt_dgemm(op(A, "N", m, k), op(B, "N", k, n), 1.0, 0.0, C[:m, :n], 16)
        hi, lo = dd_reference("N", "N", m, n, k, 1.0, A, lda, B, ldb, 0.0, C, ldc)
        assert rel_error_vs_dd(out, hi, lo) <= U64
        assert 2 * info["max_abs_cprime"] < M.modulus_product(16)


def _crt_weights(n, mods):
    P = math.prod(mods[:n])
    W = []
    for p in mods[:n]:
        Mp = P // p
        W.append(Mp * pow(Mp % p, -1, p))
    return P, W


def test_residue_route_reconstructs_the_exact_product():
    """Symmetric residues of A', B' multiplied mod p and recombined with the weights
    W_l = (P/p_l)((P/p_l)^-1 mod p_l) give C' exactly: the device's arithmetic, in
    Python integers."""
    M = crt_model()
    rng = np.random.default_rng(7)
    m, n, k = 12, 9, 40
    A = rng.uniform(-1, 1, (m, k)) * 2.0 ** rng.integers(-8, 9, (m, k))
    B = rng.uniform(-1, 1, (n, k))
    for nmod in (8, 16, 20):
        b = M.bits(nmod)
        _, Ai = M.scaled_integers(A, b)
        _, Bi = M.scaled_integers(B, b)
        exact = Ai.dot(Bi.T)
        P, W = _crt_weights(nmod, M.MODULI)
        S = np.zeros((m, n), dtype=object)
        for p, w in zip(M.MODULI[:nmod], W):
            hi = p // 2 - (0 if p % 2 else 1)

            def sym(v):
                r = int(v) % p
                return r - p if r > hi else r

            ra = np.vectorize(sym, otypes=[object])(Ai)
            rb = np.vectorize(sym, otypes=[object])(Bi)
            assert all(-128 <= int(v) <= 127 for v in ra.ravel())
            cr = np.vectorize(lambda v: int(v) % p, otypes=[object])(ra.dot(rb.T))
            S = S + cr * w
        for i in range(m):
            for j in range(n):
                R = int(S[i, j]) % P
                if R > P // 2:
                    R -= P
                assert R == int(exact[i, j])
