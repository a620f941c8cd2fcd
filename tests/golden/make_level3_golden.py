"""Generates tests/golden/level3_golden.npz from the REFERENCE implementation.

Runs Eigen's own ?gemmtr_, ?syrk_, ?syr2k_, ?symm_, ?trmm_ and ?trsm_ (blas/level3_impl.h:98-754),
compiled from the reference sources into oracle/_ref/libeigen_ref_blas.so by ``make -C oracle ref``,
on seeded inputs and records inputs and outputs.  A strong xerbla_ recorder
(oracle/librecord_xerbla.so) is loaded first so the argument-error info codes and routine names are
captured instead of printed.

Cases, for double and single precision
  * every combination of the character arguments (side, uplo, trans, diag) on sizes from the netlib
    Level-3 tester's grid (blas/testing/dblat3.dat: {0,1,2,3,5,9}) plus a 33 x 17 case, with padded
    leading dimensions and alpha/beta from {0, 0.7, 1, 1.3} (every pair on the 5 x 9 case);
  * entries the routine must not read hold NaN: the unused triangle of A (symm, trmm, trsm), the
    stored diagonal when diag = 'U', and the other triangle of C (gemmtr, syrk, syr2k), which must
    come back bit for bit;
  * beta == 0 with NaN in C's triangle (overwritten);
  * argument errors, one per info code of each routine.

    python tests/golden/make_level3_golden.py
"""
from __future__ import annotations

import ctypes
import itertools
import json
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
OUT = Path(__file__).resolve().parent / "level3_golden.npz"

# argument kinds of each routine, in order: c = character, i = dimension, s = scalar,
# a = array (input), o = array (output)
SIGNATURES = {
    "gemmtr": "cccii" "s" "ai" "ai" "s" "oi",
    "syrk": "ccii" "s" "ai" "s" "oi",
    "syr2k": "ccii" "s" "ai" "ai" "s" "oi",
    "symm": "ccii" "s" "ai" "ai" "s" "oi",
    "trmm": "ccccii" "s" "ai" "oi",
    "trsm": "ccccii" "s" "ai" "oi",
}


def fortran_args(kinds: str, values, ctype, itype=ctypes.c_int):
    """ctypes arguments of a Fortran-convention BLAS call (everything by reference)."""
    out, keep = [], []
    for kind, v in zip(kinds, values):
        if kind == "c":
            out.append(ctypes.c_char_p(v.encode()))
        elif kind == "i":
            x = itype(v)
            keep.append(x)
            out.append(ctypes.byref(x))
        elif kind == "s":
            x = ctype(v)
            keep.append(x)
            out.append(ctypes.cast(ctypes.byref(x), ctypes.c_void_p))
        else:
            out.append(ctypes.c_void_p(v if isinstance(v, int) else (int(v.ctypes.data) if v is not None else 0)))
    return out, keep


def load_reference():
    rec = ctypes.CDLL(str(ROOT / "oracle" / "librecord_xerbla.so"), mode=ctypes.RTLD_GLOBAL)
    ref = ctypes.CDLL(str(ROOT / "oracle" / "_ref" / "libeigen_ref_blas.so"), mode=ctypes.RTLD_GLOBAL)
    rec.record_xerbla_last_info.restype = ctypes.c_int
    rec.record_xerbla_calls.restype = ctypes.c_int
    rec.record_xerbla_last_name.restype = ctypes.c_char_p
    return rec, ref


def call(lib, dtype: str, routine: str, values, ilp64: bool = False) -> None:
    ctype = ctypes.c_double if dtype == "d" else ctypes.c_float
    args, keep = fortran_args(SIGNATURES[routine], values, ctype, ctypes.c_int64 if ilp64 else ctypes.c_int)
    getattr(lib, dtype + routine + ("_64_" if ilp64 else "_"))(*args)
    del keep


def _tri_mask(n: int, upper: bool) -> np.ndarray:
    return np.triu(np.ones((n, n), bool)) if upper else np.tril(np.ones((n, n), bool))


def make_case(rng, dtype, routine, chars, dims, alpha, beta, pad, special=None):
    """Inputs of one case as a dict of Fortran-ordered arrays plus its argument list."""
    npdt = np.float64 if dtype == "d" else np.float32

    def mat(rows, cols):
        return np.asfortranarray(rng.uniform(-1, 1, (max(1, rows + pad), max(1, cols))).astype(npdt))

    arrays = {}
    given, chars = chars, tuple(c.upper() for c in chars)  # the call gets the characters as given
    if routine in ("gemmtr", "syrk", "syr2k"):
        uplo = chars[0]
        n, k = dims
        upper = uplo == "U"
        if routine == "gemmtr":
            ta, tb = chars[1], chars[2]
            A = mat(*((n, k) if ta == "N" else (k, n)))
            B = mat(*((k, n) if tb == "N" else (n, k)))
        else:
            tr = chars[1]
            A = mat(*((n, k) if tr == "N" else (k, n)))
            B = mat(*((n, k) if tr == "N" else (k, n))) if routine == "syr2k" else None
        C = mat(n, n)
        if n:
            C[:n, :n][~_tri_mask(n, upper)] = np.nan  # the other triangle: never touched
        if special == "nan_c" and n:
            C[0, n - 1 if upper else 0] = np.nan
        arrays.update(A=A, C=C)
        if B is not None:
            arrays["B"] = B
        lda, ldc = A.shape[0], C.shape[0]
        if routine == "gemmtr":
            values = [*given, n, k, alpha, A, lda, B, B.shape[0], beta, C, ldc]
        elif routine == "syrk":
            values = [*given, n, k, alpha, A, lda, beta, C, ldc]
        else:
            values = [*given, n, k, alpha, A, lda, B, B.shape[0], beta, C, ldc]
    elif routine == "symm":
        side, uplo = chars
        m, n = dims
        size = m if side == "L" else n
        A, B, C = mat(size, size), mat(m, n), mat(m, n)
        if size:
            A[:size, :size][~_tri_mask(size, uplo == "U")] = np.nan  # unused triangle
        if special == "nan_c" and m and n:
            C[0, 0] = np.nan
        arrays.update(A=A, B=B, C=C)
        values = [*given, m, n, alpha, A, A.shape[0], B, B.shape[0], beta, C, C.shape[0]]
    else:
        side, uplo, tr, diag = chars
        m, n = dims
        size = m if side == "L" else n
        A, B = mat(size, size), mat(m, n)
        if size:
            sq = A[:size, :size]
            tri = _tri_mask(size, uplo == "U")
            if routine == "trsm":  # well conditioned: small off-diagonal, diagonal away from 0
                sq *= 1.0 / size
                np.fill_diagonal(sq, rng.choice([-1.0, 1.0], size) * rng.uniform(1.0, 2.0, size))
            sq[~tri] = np.nan  # unused triangle
            if diag == "U":
                np.fill_diagonal(sq, np.nan)  # the unit diagonal is not read
        arrays.update(A=A, B=B)
        values = [*given, m, n, alpha, A, A.shape[0], B, B.shape[0]]
    return arrays, values


def main() -> None:
    rec, ref = load_reference()
    rng = np.random.default_rng(20240601)
    arrays: dict[str, np.ndarray] = {}
    meta = []
    sizes = [(0, 3), (3, 0), (1, 1), (2, 3), (5, 9), (9, 5), (33, 17)]
    full = {(5, 9)}  # every alpha/beta pair on these

    def record(dtype, routine, chars, dims, alpha, beta, pad, special=None):
        ins, values = make_case(rng, dtype, routine, chars, dims, alpha, beta, pad, special)
        before = {k: v.copy(order="F") for k, v in ins.items()}
        call(ref, dtype, routine, values)
        out_name = "C" if routine in ("gemmtr", "syrk", "syr2k", "symm") else "B"
        idx = len(meta)
        for k, v in before.items():
            arrays[f"{k}{idx}"] = v
        arrays[f"out{idx}"] = ins[out_name]
        meta.append(dict(dtype=dtype, routine=routine, chars="".join(chars), dims=list(dims), alpha=alpha, beta=beta,
                         special=special))

    for dtype in ("d", "s"):
        for dims in sizes:
            pairs = [(1.0, 0.0), (0.7, 1.3), (0.0, 1.3), (0.7, 1.0)] if dims in full else [(0.7, 1.3)]
            for uplo, ta, tb in itertools.product("UL", "NT", "NT"):
                for alpha, beta in pairs:
                    record(dtype, "gemmtr", (uplo, ta, tb), dims, alpha, beta, 1)
            for routine in ("syrk", "syr2k"):
                for uplo, tr in itertools.product("UL", "NTC"):
                    for alpha, beta in pairs:
                        record(dtype, routine, (uplo, tr), dims, alpha, beta, 1)
            for side, uplo in itertools.product("LR", "UL"):
                for alpha, beta in pairs:
                    record(dtype, "symm", (side, uplo), dims, alpha, beta, 2)
            alphas = [1.0, 0.7, -1.3] if dims in full else [0.7]
            for routine in ("trmm", "trsm"):
                for side, uplo, tr, diag in itertools.product("LR", "UL", "NTC", "NU"):
                    for alpha in alphas:
                        record(dtype, routine, (side, uplo, tr, diag), dims, alpha, 0.0, 1)
        record(dtype, "syrk", ("U", "N"), (9, 5), 0.7, 0.0, 1, special="nan_c")
        record(dtype, "gemmtr", ("L", "T", "N"), (9, 5), 0.7, 0.0, 1, special="nan_c")
        record(dtype, "symm", ("R", "L"), (9, 5), 0.7, 0.0, 1, special="nan_c")
        # lower-case characters are accepted like upper-case ones
        record(dtype, "trsm", ("l", "u", "t", "n"), (9, 5), 0.7, 0.0, 1)
        record(dtype, "syrk", ("l", "c"), (9, 5), 0.7, 1.3, 1)

    # argument errors: each routine's argument list with one bad entry per info code
    dummy = np.zeros(256)
    err_cases = {
        "gemmtr": [("XNN", 2, 2, 2, 2, 2), ("UQN", 2, 2, 2, 2, 2), ("UNQ", 2, 2, 2, 2, 2), ("UNN", -1, 2, 2, 2, 2),
                   ("UNN", 2, -1, 2, 2, 2), ("UNN", 3, 2, 2, 2, 3), ("UTN", 2, 3, 2, 3, 2), ("UNN", 2, 3, 2, 2, 2),
                   ("UNT", 3, 2, 3, 2, 3), ("UNN", 3, 2, 3, 2, 2), ("lnn", 0, 0, 1, 1, 1)],
        "syrk": [("XN", 2, 2, 2, 2), ("UQ", 2, 2, 2, 2), ("UN", -1, 2, 2, 2), ("UN", 2, -1, 2, 2), ("UN", 3, 2, 2, 3),
                 ("UT", 2, 3, 2, 2), ("UN", 3, 2, 3, 2), ("uc", 0, 0, 1, 1)],
        "syr2k": [("XN", 2, 2, 2, 2, 2), ("UQ", 2, 2, 2, 2, 2), ("UN", -1, 2, 2, 2, 2), ("UN", 2, -1, 2, 2, 2),
                  ("UN", 3, 2, 2, 3, 3), ("UN", 3, 2, 3, 2, 3), ("UT", 2, 3, 3, 2, 2), ("UN", 3, 2, 3, 3, 2)],
        "symm": [("XU", 2, 2, 2, 2, 2), ("LX", 2, 2, 2, 2, 2), ("LU", -1, 2, 2, 2, 2), ("LU", 2, -1, 2, 2, 2),
                 ("LU", 3, 2, 2, 3, 3), ("RU", 2, 3, 2, 2, 2), ("LU", 3, 2, 3, 2, 3), ("LU", 3, 2, 3, 3, 2),
                 ("rl", 0, 0, 1, 1, 1)],
        "trmm": [("XUNN", 2, 2, 2, 2), ("LXNN", 2, 2, 2, 2), ("LUXN", 2, 2, 2, 2), ("LUNX", 2, 2, 2, 2),
                 ("LUNN", -1, 2, 2, 2), ("LUNN", 2, -1, 2, 2), ("LUNN", 3, 2, 2, 3), ("RUNN", 2, 3, 2, 2),
                 ("LUNN", 3, 2, 3, 2), ("rltu", 0, 0, 1, 1)],
    }
    err_cases["trsm"] = err_cases["trmm"]
    err_meta = []
    for routine, cases in err_cases.items():
        for case in cases:
            chars, dims = case[0], case[1:]
            if routine == "gemmtr":
                n, k, lda, ldb, ldc = dims
                values = [*chars, n, k, 1.0, dummy, lda, dummy, ldb, 0.0, dummy, ldc]
            elif routine == "syrk":
                n, k, lda, ldc = dims
                values = [*chars, n, k, 1.0, dummy, lda, 0.0, dummy, ldc]
            elif routine in ("syr2k", "symm"):
                a, b, lda, ldb, ldc = dims
                values = [*chars, a, b, 1.0, dummy, lda, dummy, ldb, 0.0, dummy, ldc]
            else:
                m, n, lda, ldb = dims
                values = [*chars, m, n, 1.0, dummy, lda, dummy, ldb]
            rec.record_xerbla_reset()
            call(ref, "d", routine, values)
            info = int(rec.record_xerbla_last_info()) if rec.record_xerbla_calls() else 0
            name = rec.record_xerbla_last_name().decode() if info else ""
            err_meta.append(dict(routine=routine, values=[v if not isinstance(v, np.ndarray) else None for v in values],
                                 info=info, name=name))
    arrays["meta"] = np.frombuffer(json.dumps({"cases": meta, "errors": err_meta}).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **arrays)
    print(f"wrote {OUT} ({len(meta)} cases, {len(err_meta)} argument cases)")


if __name__ == "__main__":
    main()
