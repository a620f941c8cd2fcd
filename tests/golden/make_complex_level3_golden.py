"""Generates tests/golden/complex_level3_golden.npz from the REFERENCE implementation.

Runs Eigen's own z/c trsm_, trmm_, symm_ and hemm_ (blas/level3_impl.h:230-592 and :760-831 for
std::complex), compiled from the reference sources into oracle/_ref/libeigen_ref_blas.so by
``make -C oracle ref``, on seeded inputs and records inputs and outputs, with a strong xerbla_
recorder (oracle/librecord_xerbla.so) loaded first for the argument errors.

Cases, for complex<double> and complex<float>
  * trsm / trmm: every (side, uplo, transa in N/T/C, diag) on sizes from the netlib tester's grid
    plus 33 x 17; trsm's triangles are well conditioned (small off-diagonal, diagonal of modulus
    1..2 with a random phase);
  * symm / hemm: every (side, uplo), alpha/beta from {0, 1, 0.7-0.3i, -1.1+0.4i};
  * NaN in every entry the routine must not read (the other triangle, a unit diagonal), and a
    nonzero imaginary part on hemm's diagonal (only its real part counts);
  * argument errors, one per info code.

    python tests/golden/make_complex_level3_golden.py
"""
from __future__ import annotations

import ctypes
import itertools
import json
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
OUT = Path(__file__).resolve().parent / "complex_level3_golden.npz"


def load_reference():
    rec = ctypes.CDLL(str(ROOT / "oracle" / "librecord_xerbla.so"), mode=ctypes.RTLD_GLOBAL)
    ref = ctypes.CDLL(str(ROOT / "oracle" / "_ref" / "libeigen_ref_blas.so"), mode=ctypes.RTLD_GLOBAL)
    rec.record_xerbla_last_info.restype = ctypes.c_int
    rec.record_xerbla_calls.restype = ctypes.c_int
    rec.record_xerbla_last_name.restype = ctypes.c_char_p
    return rec, ref


def call(lib, dtype, routine, chars, dims, alpha, A, lda, B, ldb, beta=None, C=None, ldc=None):
    real = ctypes.c_double if dtype == "z" else ctypes.c_float
    i = ctypes.c_int
    al = (real * 2)(alpha.real, alpha.imag)
    P = lambda x: ctypes.c_void_p(x.ctypes.data)  # noqa: E731
    R = ctypes.byref
    cs = [ctypes.c_char_p(c.encode()) for c in chars]
    if routine in ("trsm", "trmm"):
        getattr(lib, dtype + routine + "_")(*cs, R(i(dims[0])), R(i(dims[1])), al, P(A), R(i(lda)), P(B), R(i(ldb)))
    else:
        be = (real * 2)(beta.real, beta.imag)
        getattr(lib, dtype + routine + "_")(*cs, R(i(dims[0])), R(i(dims[1])), al, P(A), R(i(lda)), P(B), R(i(ldb)),
                                            be, P(C), R(i(ldc)))


def main() -> None:
    rec, ref = load_reference()
    rng = np.random.default_rng(20240603)
    arrays: dict[str, np.ndarray] = {}
    meta = []

    def cmat(rows, cols, npdt):
        x = rng.uniform(-1, 1, (rows, cols)) + 1j * rng.uniform(-1, 1, (rows, cols))
        return np.asfortranarray(x.astype(npdt))

    def tri_mask(n, upper):
        return np.triu(np.ones((n, n), bool)) if upper else np.tril(np.ones((n, n), bool))

    def record(dtype, routine, chars, dims, alpha, beta=None):
        npdt = np.complex128 if dtype == "z" else np.complex64
        side, uplo = chars[0].upper(), chars[1].upper()
        m, n = dims
        size = m if side == "L" else n
        A = cmat(size + 1, max(size, 1), npdt)
        B = cmat(m + 2, max(n, 1), npdt)
        C = cmat(m + 1, max(n, 1), npdt) if routine in ("symm", "hemm") else None
        if size:
            sq = A[:size, :size]
            if routine == "trsm":
                sq *= 1.0 / size
                phase = np.exp(1j * rng.uniform(0, 2 * np.pi, size))
                np.fill_diagonal(sq, (rng.uniform(1.0, 2.0, size) * phase).astype(npdt))
            sq[~tri_mask(size, uplo == "U")] = np.nan
            if routine in ("trsm", "trmm") and chars[3].upper() == "U":
                np.fill_diagonal(sq, np.nan)  # the unit diagonal is not read
            if routine == "hemm":
                np.fill_diagonal(sq, np.diag(sq).real + 0.5j)  # only the real part counts
        ins = {"A": A, "B": B} if C is None else {"A": A, "B": B, "C": C}
        before = {k: v.copy(order="F") for k, v in ins.items()}
        if C is None:
            call(ref, dtype, routine, chars, dims, alpha, A, A.shape[0], B, B.shape[0])
        else:
            call(ref, dtype, routine, chars, dims, alpha, A, A.shape[0], B, B.shape[0], beta, C, C.shape[0])
        idx = len(meta)
        for k, v in before.items():
            arrays[f"{k}{idx}"] = v
        arrays[f"out{idx}"] = ins["C" if C is not None else "B"]
        meta.append(dict(dtype=dtype, routine=routine, chars="".join(chars), dims=list(dims),
                         alpha=[alpha.real, alpha.imag], beta=None if beta is None else [beta.real, beta.imag]))

    sizes = [(0, 3), (3, 0), (1, 1), (5, 9), (9, 5), (33, 17)]
    scalars = [0j, 1 + 0j, 0.7 - 0.3j, -1.1 + 0.4j]
    for dtype in ("z", "c"):
        for dims in sizes:
            alphas = [1 + 0j, 0.7 - 0.3j, -1.1 + 0.4j] if dims == (5, 9) else [0.7 - 0.3j]
            for routine in ("trsm", "trmm"):
                for side, uplo, tr, diag in itertools.product("LR", "UL", "NTC", "NU"):
                    for alpha in alphas:
                        record(dtype, routine, (side, uplo, tr, diag), dims, alpha)
            pairs = list(itertools.product(scalars, scalars)) if dims == (5, 9) else [(0.7 - 0.3j, -1.1 + 0.4j)]
            for routine in ("symm", "hemm"):
                for side, uplo in itertools.product("LR", "UL"):
                    for alpha, beta in pairs:
                        record(dtype, routine, (side, uplo), dims, alpha, beta)
        record(dtype, "trsm", ("l", "u", "c", "n"), (9, 5), 0.7 - 0.3j)
        record(dtype, "hemm", ("r", "l"), (9, 5), 0.7 - 0.3j, 0j)

    dummy = np.zeros(256, dtype=np.complex128)
    err_cases = {
        "trsm": [("XUNN", 2, 2, 2, 2), ("LXNN", 2, 2, 2, 2), ("LUXN", 2, 2, 2, 2), ("LUNX", 2, 2, 2, 2),
                 ("LUNN", -1, 2, 2, 2), ("LUNN", 2, -1, 2, 2), ("LUCN", 3, 2, 2, 3), ("RUNN", 2, 3, 2, 2),
                 ("LUNN", 3, 2, 3, 2), ("rlcu", 0, 0, 1, 1)],
        "hemm": [("XU", 2, 2, 2, 2, 2), ("LX", 2, 2, 2, 2, 2), ("LU", -1, 2, 2, 2, 2), ("LU", 2, -1, 2, 2, 2),
                 ("LU", 3, 2, 2, 3, 3), ("RU", 2, 3, 2, 2, 2), ("LU", 3, 2, 3, 2, 3), ("LU", 3, 2, 3, 3, 2),
                 ("rl", 0, 0, 1, 1, 1)],
    }
    err_cases["trmm"] = err_cases["trsm"]
    err_cases["symm"] = err_cases["hemm"]
    err_meta = []
    for routine, cases in err_cases.items():
        for case in cases:
            chars, d = case[0], case[1:]
            rec.record_xerbla_reset()
            if routine in ("trsm", "trmm"):
                call(ref, "z", routine, chars, (d[0], d[1]), 1 + 0j, dummy, d[2], dummy, d[3])
                values = [*chars, d[0], d[1], 1.0, None, d[2], None, d[3]]
            else:
                call(ref, "z", routine, chars, (d[0], d[1]), 1 + 0j, dummy, d[2], dummy, d[3], 0j, dummy, d[4])
                values = [*chars, d[0], d[1], 1.0, None, d[2], None, d[3], 0.0, None, d[4]]
            info = int(rec.record_xerbla_last_info()) if rec.record_xerbla_calls() else 0
            err_meta.append(dict(routine=routine, values=values, info=info,
                                 name=rec.record_xerbla_last_name().decode() if info else ""))
    arrays["meta"] = np.frombuffer(json.dumps({"cases": meta, "errors": err_meta}).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **arrays)
    print(f"wrote {OUT} ({len(meta)} cases, {len(err_meta)} argument cases)")


if __name__ == "__main__":
    main()
