"""Generates tests/golden/gemm_golden.npz from the REFERENCE implementation.

Runs Eigen's own sgemm_/dgemm_ (blas/level3_impl.h:12-96), compiled from the
reference sources into oracle/_ref/libeigen_ref_blas.so by ``make -C oracle ref``,
on seeded inputs and records inputs and outputs.  A strong xerbla_ recorder
(oracle/librecord_xerbla.so) is loaded first so the argument-error info codes of
blas/level3_impl.h:61-78 are captured instead of printed.

Cases
  * the parameter grid of the netlib Level-3 tester's data file
    (blas/testing/dblat3.dat: sizes {0,1,2,3,5,9}, alpha {0,1,0.7}, beta {0,1,1.3}),
    on a subset of (m,n,k) triples, for every (transa, transb) in N/T/C;
  * larger products with padded leading dimensions (up to 64^3);
  * IEEE edge cases: alpha == 0 with NaN/Inf in A and B (C keeps beta*C, A/B unread,
    pinned by test/product_extra.cpp:665-728), beta == 0 with NaN in C (C overwritten);
  * argument errors (info 1,2,3,4,5,8,10,13).

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes
import itertools
import json
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
OUT = Path(__file__).resolve().parent / "gemm_golden.npz"


def load_reference():
    rec = ctypes.CDLL(str(ROOT / "oracle" / "librecord_xerbla.so"), mode=ctypes.RTLD_GLOBAL)
    ref = ctypes.CDLL(str(ROOT / "oracle" / "_ref" / "libeigen_ref_blas.so"), mode=ctypes.RTLD_GLOBAL)
    return rec, ref


def call(ref, name, ctype, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
    i = ctypes.c_int
    al, be = ctype(alpha), ctype(beta)
    f = getattr(ref, name)
    f(ta.encode(), tb.encode(), ctypes.byref(i(m)), ctypes.byref(i(n)), ctypes.byref(i(k)), ctypes.byref(al),
      A.ctypes.data_as(ctypes.c_void_p), ctypes.byref(i(lda)), B.ctypes.data_as(ctypes.c_void_p), ctypes.byref(i(ldb)),
      ctypes.byref(be), C.ctypes.data_as(ctypes.c_void_p), ctypes.byref(i(ldc)))


def main() -> None:
    rec, ref = load_reference()
    rec.record_xerbla_last_info.restype = ctypes.c_int
    rng = np.random.default_rng(20240531)
    arrays: dict[str, np.ndarray] = {}
    meta = []
    triples = [(0, 3, 2), (3, 0, 4), (2, 3, 0), (1, 1, 1), (2, 3, 5), (3, 5, 9), (5, 9, 3), (9, 9, 9), (9, 2, 1),
               (5, 5, 5)]
    big = [(17, 33, 65, 3), (64, 64, 64, 8), (40, 23, 31, 1)]

    def add_case(dtype, ta, tb, m, n, k, alpha, beta, pad, special=None):
        npdt = np.float64 if dtype == "d" else np.float32
        ar, ac = (k, m) if ta != "N" else (m, k)
        br, bc = (n, k) if tb != "N" else (k, n)
        lda, ldb, ldc = max(1, ar + pad), max(1, br + pad), max(1, m + pad)
        A = np.asfortranarray(rng.uniform(-1, 1, (lda, max(ac, 1))).astype(npdt))
        B = np.asfortranarray(rng.uniform(-1, 1, (ldb, max(bc, 1))).astype(npdt))
        C = np.asfortranarray(rng.uniform(-1, 1, (ldc, max(n, 1))).astype(npdt))
        if special == "nan_ab":
            A[0, 0] = np.nan
            B[-1, -1] = np.inf
        if special == "nan_c":
            C[0, 0] = np.nan
            C[-1, -1] = -np.inf
        Cin = C.copy(order="F")
        call(ref, "dgemm_" if dtype == "d" else "sgemm_", ctypes.c_double if dtype == "d" else ctypes.c_float, ta, tb,
             m, n, k, alpha, A, lda, B, ldb, beta, C, ldc)
        idx = len(meta)
        arrays[f"A{idx}"], arrays[f"B{idx}"], arrays[f"Cin{idx}"], arrays[f"Cout{idx}"] = A, B, Cin, C
        meta.append(dict(dtype=dtype, ta=ta, tb=tb, m=m, n=n, k=k, alpha=alpha, beta=beta, lda=lda, ldb=ldb, ldc=ldc,
                         special=special))

    for dtype in ("d", "s"):
        for ta, tb in itertools.product("NTC", "NTC"):
            for (m, n, k) in triples:
                for alpha, beta in itertools.product((0.0, 1.0, 0.7), (0.0, 1.0, 1.3)):
                    if (m, n, k) not in ((2, 3, 5), (9, 9, 9)) and (alpha, beta) not in ((1.0, 0.0), (0.7, 1.3)):
                        continue
                    add_case(dtype, ta, tb, m, n, k, alpha, beta, pad=1)
        for ta, tb in (("N", "N"), ("N", "T"), ("T", "N")):
            for (m, n, k, pad) in big:
                add_case(dtype, ta, tb, m, n, k, 1.5, 0.5, pad)
        add_case(dtype, "N", "N", 7, 6, 5, 0.0, 1.3, 2, special="nan_ab")
        add_case(dtype, "T", "N", 7, 6, 5, 0.0, 0.0, 2, special="nan_ab")
        add_case(dtype, "N", "T", 7, 6, 5, 1.0, 0.0, 2, special="nan_c")
        add_case(dtype, "N", "N", 7, 6, 5, 0.7, 1.0, 2, special="nan_c")

    # argument errors: (ta, tb, m, n, k, lda, ldb, ldc)
    err_cases = [("X", "N", 2, 2, 2, 2, 2, 2), ("N", "Q", 2, 2, 2, 2, 2, 2), ("N", "N", -1, 2, 2, 2, 2, 2),
                 ("N", "N", 2, -1, 2, 2, 2, 2), ("N", "N", 2, 2, -1, 2, 2, 2), ("N", "N", 3, 2, 2, 2, 2, 3),
                 ("T", "N", 2, 2, 3, 2, 3, 2), ("N", "N", 2, 2, 3, 2, 2, 2), ("N", "T", 2, 3, 2, 2, 2, 2),
                 ("N", "N", 3, 2, 2, 3, 2, 2), ("n", "t", 0, 0, 0, 1, 1, 1), ("c", "C", 0, 0, 0, 0, 1, 1),
                 ("N", "N", 0, 0, 0, 0, 0, 0)]
    err_meta = []
    dummy = np.zeros(64)
    for (ta, tb, m, n, k, lda, ldb, ldc) in err_cases:
        rec.record_xerbla_reset()
        call(ref, "dgemm_", ctypes.c_double, ta, tb, m, n, k, 1.0, dummy, lda, dummy, ldb, 0.0, dummy, ldc)
        err_meta.append(dict(ta=ta, tb=tb, m=m, n=n, k=k, lda=lda, ldb=ldb, ldc=ldc,
                             info=int(rec.record_xerbla_last_info()) if rec.record_xerbla_calls() else 0))
    arrays["meta"] = np.frombuffer(json.dumps({"cases": meta, "errors": err_meta}).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **arrays)
    print(f"wrote {OUT} ({len(meta)} product cases, {len(err_meta)} argument cases)")


if __name__ == "__main__":
    main()
