"""Generates tests/golden/complex_golden.npz from the REFERENCE implementation.

Runs Eigen's own zgemm_ / cgemm_ (blas/level3_impl.h:12-96 instantiated for std::complex by
blas/complex_double.cpp and blas/complex_single.cpp), compiled from the reference sources into
oracle/_ref/libeigen_ref_blas.so by ``make -C oracle ref``, on seeded inputs and records inputs
and outputs.  A strong xerbla_ recorder (oracle/librecord_xerbla.so) is loaded first so the
argument-error info codes are captured instead of printed.

Cases, for complex<double> and complex<float>
  * every (transa, transb) in N/T/C on sizes from the netlib Level-3 tester's grid
    (blas/testing/zblat3.dat: {0,1,2,3,5,9}) plus 33 x 17 x 40, padded leading dimensions,
    alpha/beta from {0, 1, 0.7-0.3i, -1.1+0.4i};
  * alpha == 0 with NaN in A and B (A and B unread), beta == 0 with NaN in C (overwritten);
  * argument errors (info 1,2,3,4,5,8,10,13).

    python tests/golden/make_complex_golden.py
"""
from __future__ import annotations

import ctypes
import itertools
import json
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
OUT = Path(__file__).resolve().parent / "complex_golden.npz"


def load_reference():
    rec = ctypes.CDLL(str(ROOT / "oracle" / "librecord_xerbla.so"), mode=ctypes.RTLD_GLOBAL)
    ref = ctypes.CDLL(str(ROOT / "oracle" / "_ref" / "libeigen_ref_blas.so"), mode=ctypes.RTLD_GLOBAL)
    rec.record_xerbla_last_info.restype = ctypes.c_int
    rec.record_xerbla_calls.restype = ctypes.c_int
    rec.record_xerbla_last_name.restype = ctypes.c_char_p
    return rec, ref


def call(lib, dtype, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
    """zgemm_ (dtype "z") or cgemm_ ("c") with complex alpha, beta and complex arrays."""
    real = ctypes.c_double if dtype == "z" else ctypes.c_float
    i = ctypes.c_int
    al = (real * 2)(alpha.real, alpha.imag)
    be = (real * 2)(beta.real, beta.imag)
    getattr(lib, dtype + "gemm_")(ta.encode(), tb.encode(), ctypes.byref(i(m)), ctypes.byref(i(n)),
                                   ctypes.byref(i(k)), al, ctypes.c_void_p(A.ctypes.data), ctypes.byref(i(lda)),
                                   ctypes.c_void_p(B.ctypes.data), ctypes.byref(i(ldb)), be,
                                   ctypes.c_void_p(C.ctypes.data), ctypes.byref(i(ldc)))


def main() -> None:
    rec, ref = load_reference()
    rng = np.random.default_rng(20240602)
    arrays: dict[str, np.ndarray] = {}
    meta = []

    def cmat(rows, cols, npdt):
        x = rng.uniform(-1, 1, (rows, cols)) + 1j * rng.uniform(-1, 1, (rows, cols))
        return np.asfortranarray(x.astype(npdt))

    def add(dtype, ta, tb, m, n, k, alpha, beta, pad, special=None):
        npdt = np.complex128 if dtype == "z" else np.complex64
        ar, ac = (k, m) if ta != "N" else (m, k)
        br, bc = (n, k) if tb != "N" else (k, n)
        lda, ldb, ldc = max(1, ar + pad), max(1, br + pad), max(1, m + pad)
        A, B, C = cmat(lda, max(ac, 1), npdt), cmat(ldb, max(bc, 1), npdt), cmat(ldc, max(n, 1), npdt)
        if special == "nan_ab":
            A[0, 0] = np.nan
            B[-1, -1] = complex(np.inf, 1.0)
        if special == "nan_c":
            C[0, 0] = complex(np.nan, 0.0)
        Cin = C.copy(order="F")
        call(ref, dtype, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc)
        idx = len(meta)
        arrays[f"A{idx}"], arrays[f"B{idx}"], arrays[f"Cin{idx}"], arrays[f"Cout{idx}"] = A, B, Cin, C
        meta.append(dict(dtype=dtype, ta=ta, tb=tb, m=m, n=n, k=k, alpha=[alpha.real, alpha.imag],
                         beta=[beta.real, beta.imag], lda=lda, ldb=ldb, ldc=ldc, special=special))

    scalars = [0j, 1 + 0j, 0.7 - 0.3j, -1.1 + 0.4j]
    triples = [(0, 3, 2), (3, 0, 4), (2, 3, 0), (1, 1, 1), (2, 3, 5), (5, 9, 3), (9, 5, 9), (33, 17, 40)]
    for dtype in ("z", "c"):
        for ta, tb in itertools.product("NTC", "NTC"):
            for (m, n, k) in triples:
                pairs = itertools.product(scalars, scalars) if (m, n, k) == (9, 5, 9) else [(0.7 - 0.3j, -1.1 + 0.4j)]
                for alpha, beta in pairs:
                    add(dtype, ta, tb, m, n, k, alpha, beta, pad=1)
        add(dtype, "N", "C", 7, 6, 5, 0j, 0.7 - 0.3j, 2, special="nan_ab")
        add(dtype, "C", "N", 7, 6, 5, 0j, 0j, 2, special="nan_ab")
        add(dtype, "T", "C", 7, 6, 5, 1 + 0j, 0j, 2, special="nan_c")
        add(dtype, "n", "c", 7, 6, 5, 0.7 - 0.3j, 1 + 0j, 2)

    err_cases = [("X", "N", 2, 2, 2, 2, 2, 2), ("N", "Q", 2, 2, 2, 2, 2, 2), ("N", "N", -1, 2, 2, 2, 2, 2),
                 ("N", "N", 2, -1, 2, 2, 2, 2), ("N", "N", 2, 2, -1, 2, 2, 2), ("N", "N", 3, 2, 2, 2, 2, 3),
                 ("C", "N", 2, 2, 3, 2, 3, 2), ("N", "N", 2, 2, 3, 2, 2, 2), ("N", "C", 2, 3, 2, 2, 2, 2),
                 ("N", "N", 3, 2, 2, 3, 2, 2), ("c", "t", 0, 0, 0, 1, 1, 1)]
    err_meta = []
    dummy = np.zeros(64, dtype=np.complex128)
    for (ta, tb, m, n, k, lda, ldb, ldc) in err_cases:
        rec.record_xerbla_reset()
        call(ref, "z", ta, tb, m, n, k, 1 + 0j, dummy, lda, dummy, ldb, 0j, dummy, ldc)
        info = int(rec.record_xerbla_last_info()) if rec.record_xerbla_calls() else 0
        err_meta.append(dict(ta=ta, tb=tb, m=m, n=n, k=k, lda=lda, ldb=ldb, ldc=ldc, info=info,
                             name=rec.record_xerbla_last_name().decode() if info else ""))
    arrays["meta"] = np.frombuffer(json.dumps({"cases": meta, "errors": err_meta}).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **arrays)
    print(f"wrote {OUT} ({len(meta)} product cases, {len(err_meta)} argument cases)")


if __name__ == "__main__":
    main()
