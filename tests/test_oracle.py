"""Pins the CPU oracle (oracle/oracle_gemm.c) against the reference.

* golden fixtures produced by Eigen's own sgemm_/dgemm_ (tests/golden/make_golden.py);
* the reference library itself when oracle/_ref was built here;
* the double-double GEMM against exact rational arithmetic;
* the Ozaki digit split against its defining identity.
All CPU-only.
"""
from __future__ import annotations

import ctypes
from fractions import Fraction
from pathlib import Path

import numpy as np
import pytest

from _helpers import (P, U64, ch, check_against_reference, dd_reference, gemm_error_bound, golden, make_operands,
                      oracle, op, load_xerbla_recorder, ROOT)


def _run_oracle(case):
    lib = oracle()
    C = case["Cin"].copy(order="F")
    f = lib.oracle_dgemm if case["dtype"] == "d" else lib.oracle_sgemm
    info = f(ch(case["ta"]), ch(case["tb"]), case["m"], case["n"], case["k"], case["alpha"], P(case["A"]),
             case["lda"], P(case["B"]), case["ldb"], case["beta"], P(C), case["ldc"])
    return info, C


def test_golden_fixture_count():
    cases, errors = golden()
    assert len(cases) > 600 and len(errors) == 13


@pytest.mark.parametrize("dtype", ["d", "s"])
def test_oracle_matches_golden(dtype):
    cases, _ = golden()
    n = 0
    for case in cases:
        if case["dtype"] != dtype:
            continue
        info, C = _run_oracle(case)
        assert info == 0
        check_against_reference(case, C)
        n += 1
    assert n > 300


def test_oracle_info_codes_match_golden():
    _, errors = golden()
    lib = oracle()
    for e in errors:
        assert lib.oracle_gemm_info(ch(e["ta"]), ch(e["tb"]), e["m"], e["n"], e["k"], e["lda"], e["ldb"],
                                    e["ldc"]) == e["info"], e


REF_SO = ROOT / "oracle" / "_ref" / "libeigen_ref_blas.so"


@pytest.mark.skipif(not REF_SO.exists(), reason="reference BLAS not built (make -C oracle ref)")
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T"), ("C", "n")])
def test_oracle_matches_reference_live(ta, tb):
    load_xerbla_recorder()
    ref = ctypes.CDLL(str(REF_SO), mode=ctypes.RTLD_GLOBAL)
    m, n, k = 67, 45, 130
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, ta, tb, pad=3, seed=7)
    Cref = C.copy(order="F")
    Cor = C.copy(order="F")
    i = ctypes.c_int
    al, be = ctypes.c_double(1.5), ctypes.c_double(0.5)
    ref.dgemm_(ch(ta), ch(tb), ctypes.byref(i(m)), ctypes.byref(i(n)), ctypes.byref(i(k)), ctypes.byref(al), P(A),
               ctypes.byref(i(lda)), P(B), ctypes.byref(i(ldb)), ctypes.byref(be), P(Cref), ctypes.byref(i(ldc)))
    oracle().oracle_dgemm(ch(ta), ch(tb), m, n, k, 1.5, P(A), lda, P(B), ldb, 0.5, P(Cor), ldc)
    bound = gemm_error_bound(A, ta, B, tb, m, n, k, 1.5, 0.5, C, U64)
    assert np.all(np.abs(Cor[:m, :n] - Cref[:m, :n]) <= bound)


def test_reference_xerbla_recorded_for_bad_args():
    if not REF_SO.exists():
        pytest.skip("reference BLAS not built")
    rec = load_xerbla_recorder()
    ref = ctypes.CDLL(str(REF_SO), mode=ctypes.RTLD_GLOBAL)
    rec.record_xerbla_reset()
    i = ctypes.c_int
    z = np.zeros(4)
    one = ctypes.c_double(1.0)
    ref.dgemm_(b"N", b"N", ctypes.byref(i(3)), ctypes.byref(i(2)), ctypes.byref(i(2)), ctypes.byref(one), P(z),
               ctypes.byref(i(2)), P(z), ctypes.byref(i(2)), ctypes.byref(one), P(z), ctypes.byref(i(3)))
    assert rec.record_xerbla_last_info() == 8
    assert rec.record_xerbla_last_name().decode() == "DGEMM "


def test_double_double_is_exact_on_rationals():
    """The double-double GEMM against exact Fraction arithmetic on a small product."""
    m, n, k = 5, 4, 300
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, "N", "T", pad=1, r=20, seed=3)
    hi, lo = dd_reference("N", "T", m, n, k, 1.0, A, lda, B, ldb, 0.0, None, ldc)
    a, b = op(A, "N", m, k), op(B, "T", k, n)
    for i in range(m):
        for j in range(n):
            exact = sum(Fraction(float(a[i, l])) * Fraction(float(b[l, j])) for l in range(k))
            got = Fraction(float(hi[i, j])) + Fraction(float(lo[i, j]))
            scale = sum(abs(Fraction(float(a[i, l])) * Fraction(float(b[l, j]))) for l in range(k))
            assert abs(got - exact) <= scale * Fraction(2) ** -100


def test_test_ratio_accepts_oracle_and_rejects_perturbation():
    """The restated DMMCH ratio (blas/testing/dblat3.f:2510-2621) is < 16 for a correct
    result and flags a result perturbed by 1e-9 relative."""
    lib = oracle()
    m, n, k = 9, 7, 33
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, "T", "N", pad=2, seed=5)
    Cout = C.copy(order="F")
    lib.oracle_dgemm(b"T", b"N", m, n, k, 0.7, P(A), lda, P(B), ldb, 1.3, P(Cout), ldc)
    r = lib.oracle_dgemm_test_ratio(b"T", b"N", m, n, k, 0.7, P(A), lda, P(B), ldb, 1.3, P(C), ldc, P(Cout), ldc, U64)
    assert r < 16.0
    bad = Cout.copy(order="F")
    bad[2, 3] *= 1 + 1e-9
    r2 = lib.oracle_dgemm_test_ratio(b"T", b"N", m, n, k, 0.7, P(A), lda, P(B), ldb, 1.3, P(C), ldc, P(bad), ldc, U64)
    assert r2 > 16.0


@pytest.mark.parametrize("s,r", [(4, 0), (8, 0), (9, 32), (12, 8)])
def test_ozaki_split_identity(s, r):
    """x = 2^e * sum_p d_p 2^(-6-7(p-1)) + rem, |rem| <= 2^(e-7s), |d_p| <= 64."""
    rows, cols = 37, 70
    rng = np.random.default_rng(s * 100 + r)
    X = np.asfortranarray(rng.uniform(-1, 1, (rows, cols)) * 2.0 ** rng.integers(-r, r + 1, (rows, cols)))
    X[5, :] = 0.0
    digits = np.zeros((s, rows, cols), dtype=np.int8)
    exps = np.zeros(rows, dtype=np.int32)
    oracle().oracle_ozaki_split(P(X), rows, cols, 1, rows, s, P(digits), rows, cols, P(exps))
    assert np.abs(digits.astype(int)).max() <= 64
    assert exps[5] == 0 and not digits[:, 5, :].any()
    w = np.array([2.0 ** (-6 - 7 * p) for p in range(s)])
    recon = np.einsum("p,prc->rc", w, digits.astype(np.float64)) * np.ldexp(1.0, exps)[:, None]
    bound = np.ldexp(1.0, exps - 7 * s)[:, None]
    assert np.all(np.abs(recon - X) <= bound * 1.0000001)
    mx = np.abs(X).max(axis=1)
    nz = mx > 0
    assert np.all(mx[nz] < np.ldexp(1.0, exps[nz])) and np.all(mx[nz] >= np.ldexp(1.0, exps[nz] - 1))


def test_ozaki_split_nonfinite_row():
    X = np.asfortranarray(np.ones((3, 4)))
    X[1, 2] = np.nan
    digits = np.zeros((3, 3, 4), dtype=np.int8)
    exps = np.zeros(3, dtype=np.int32)
    oracle().oracle_ozaki_split(P(X), 3, 4, 1, 3, 3, P(digits), 3, 4, P(exps))
    assert exps[1] == np.iinfo(np.int32).min and not digits[:, 1, :].any()
    assert exps[0] == 1 and exps[2] == 1


@pytest.mark.parametrize("s,r,expect", [(7, 0, 1e-14), (9, 8, 5e-16), (10, 32, 5e-16)])
def test_ozaki_model_converges(s, r, expect):
    """The oracle's Ozaki model approaches the double-double product as slices grow."""
    m, n, k = 24, 20, 300
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, "N", "N", pad=1, r=r, seed=11)
    Cm = C.copy(order="F")
    oracle().oracle_ozaki_dgemm(b"N", b"N", m, n, k, 1.0, P(A), lda, P(B), ldb, 0.0, P(Cm), ldc, s)
    hi, lo = dd_reference("N", "N", m, n, k, 1.0, A, lda, B, ldb, 0.0, None, ldc)
    err = np.linalg.norm((Cm[:m, :n] - hi) - lo) / np.linalg.norm(hi)
    assert err < expect
