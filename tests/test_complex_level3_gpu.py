"""Complex trsm_, trmm_, symm_ and hemm_ on the GPU through the C ABI, against Eigen's own
routines (blas/level3_impl.h:230-592 and :760-831 for std::complex).

* every golden case recorded from the reference (tests/golden/complex_level3_golden.npz: all
  character arguments with conjugate transposes, complex alpha/beta edge values, NaN in every
  entry the routine must not read, an imaginary part on hemm's diagonal that must be ignored):
  trmm / symm / hemm within the product error bound of the reference's result, trsm's residual
  within the same bound, padding rows untouched, for both precisions;
* sizes that recurse (trsm down to 128-row diagonal blocks) against the reference library.

Bound: lam*sqrt(k+2)*u*(|alpha| |X||Y| + |beta| |C|) per entry with complex moduli, lam = 8;
for trsm the same bound on the residual op(A) X - alpha B with |op(A)||X| + |alpha B|.
"""
from __future__ import annotations

import ctypes
import json
from pathlib import Path

import numpy as np
import pytest

import eigen_b200 as eb
from _helpers import ORACLE_DIR, U32, U64

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
GOLDEN = Path(__file__).resolve().parent / "golden" / "complex_level3_golden.npz"
REF_BLAS = ORACLE_DIR / "_ref" / "libeigen_ref_blas.so"
LAM = 8.0


@pytest.fixture(autouse=True)
def _defaults():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    eb.load()
    eb.clear_error()
    yield
    eb.set_dgemm_method(eb.METHOD_AUTO)
    eb.set_sgemm_method(eb.METHOD_AUTO)


_CASES = None


def golden_cases():
    global _CASES
    if _CASES is None:
        z = np.load(GOLDEN)
        meta = json.loads(bytes(z["meta"]).decode())
        _CASES = []
        for i, c in enumerate(meta["cases"]):
            c = dict(c)
            for k in ("A", "B", "C"):
                if f"{k}{i}" in z:
                    c[k] = z[f"{k}{i}"]
            c["out"] = z[f"out{i}"]
            c["alpha"] = complex(*c["alpha"])
            c["beta"] = None if c["beta"] is None else complex(*c["beta"])
            _CASES.append(c)
    return _CASES


def args_for(c, mats):
    m, n = c["dims"]
    if c["routine"] in ("trsm", "trmm"):
        return [*c["chars"], m, n, c["alpha"], mats["A"], c["A"].shape[0], mats["B"], c["B"].shape[0]]
    return [*c["chars"], m, n, c["alpha"], mats["A"], c["A"].shape[0], mats["B"], c["B"].shape[0], c["beta"],
            mats["C"], c["C"].shape[0]]


def run_ours(c):
    mats = {k: c[k].copy(order="F") for k in ("A", "B", "C") if k in c}
    eb.level3(c["dtype"] + c["routine"], *args_for(c, mats))
    return mats["B" if c["routine"] in ("trsm", "trmm") else "C"]


def dense_operand(c):
    """The dense op(A) (trsm / trmm) or S (symm / hemm) in complex128."""
    ch = c["chars"].upper()
    m, n = c["dims"]
    size = m if ch[0] == "L" else n
    A = c["A"][:size, :size].astype(np.complex128)
    up = ch[1] == "U"
    mask = np.triu(np.ones((size, size), bool)) if up else np.tril(np.ones((size, size), bool))
    T = np.where(mask, A, 0)
    if c["routine"] in ("trsm", "trmm"):
        if ch[3] == "U":
            np.fill_diagonal(T, 1)
        return T.conj().T if ch[2] == "C" else (T.T if ch[2] == "T" else T)
    strict = T - np.diag(np.diag(T))
    if c["routine"] == "hemm":
        return strict + strict.conj().T + np.diag(np.diag(T).real)
    return strict + strict.T + np.diag(np.diag(T))


def check(c, got, X=None):
    r, ch = c["routine"], c["chars"].upper()
    m, n = c["dims"]
    inp = c["B"] if r in ("trsm", "trmm") else c["C"]
    np.testing.assert_array_equal(got[m:, :], inp[m:, :])
    if m == 0 or n == 0:
        np.testing.assert_array_equal(got, inp)
        return
    eps = U64 if c["dtype"] == "z" else U32
    M = dense_operand(c)
    left = ch[0] == "L"
    size = m if left else n
    g = got[:m, :n].astype(np.complex128)
    B0 = c["B"][:m, :n].astype(np.complex128)
    al = c["alpha"]
    if r == "trsm":
        res = (M @ g if left else g @ M) - al * B0
        mag = (np.abs(M) @ np.abs(g) if left else np.abs(g) @ np.abs(M)) + abs(al) * np.abs(B0)
        assert np.all(np.abs(res) <= LAM * np.sqrt(size + 2) * eps * mag + 1e-300), c["chars"]
        return
    if r == "trmm":
        want = al * (M @ B0 if left else B0 @ M)
        mag = abs(al) * (np.abs(M) @ np.abs(B0) if left else np.abs(B0) @ np.abs(M))
    else:
        be = c["beta"]
        C0 = c["C"][:m, :n].astype(np.complex128)
        want = al * (M @ B0 if left else B0 @ M) + (be * C0 if be != 0 else 0)
        mag = abs(al) * (np.abs(M) @ np.abs(B0) if left else np.abs(B0) @ np.abs(M)) + abs(be) * np.abs(C0)
    bound = LAM * np.sqrt(size + 2) * eps * mag + 1e-300
    ref = c["out"][:m, :n].astype(np.complex128)
    assert np.all(np.abs(ref - want) <= bound)  # the reference meets the bound
    assert np.all(np.abs(g - want) <= bound), (c["routine"], c["chars"], float(np.max(np.abs(g - want) / bound)))


@pytest.mark.parametrize("dtype,method", [("z", eb.METHOD_NATIVE), ("z", eb.METHOD_CRT), ("c", eb.METHOD_AUTO)])
def test_golden_parity(dtype, method):
    (eb.set_dgemm_method if dtype == "z" else eb.set_sgemm_method)(method)
    count = 0
    for c in golden_cases():
        if c["dtype"] != dtype:
            continue
        got = run_ours(c)
        assert eb.last_error()[0] == eb.EB2_OK, (c["routine"], c["chars"], eb.last_error())
        check(c, got)
        count += 1
    assert count > 500


def _reference(c):
    if not REF_BLAS.exists():
        pytest.skip("oracle/_ref not built (the reference sources were absent)")
    lib = ctypes.CDLL(str(REF_BLAS), mode=ctypes.RTLD_LOCAL)
    real = ctypes.c_double if c["dtype"] == "z" else ctypes.c_float
    i = ctypes.c_int
    mats = {k: c[k].copy(order="F") for k in ("A", "B", "C") if k in c}
    out = []
    for kind, v in zip(eb.LEVEL3_SIGNATURES[c["routine"]], args_for(c, mats)):
        if kind == "c":
            out.append(ctypes.c_char_p(v.encode()))
        elif kind == "i":
            out.append(ctypes.byref(i(v)))
        elif kind == "s":
            out.append((real * 2)(complex(v).real, complex(v).imag))
        else:
            out.append(ctypes.c_void_p(v.ctypes.data))
    getattr(lib, c["dtype"] + c["routine"] + "_")(*out)
    return mats["B" if c["routine"] in ("trsm", "trmm") else "C"]


@pytest.mark.parametrize("routine,chars,dims", [("trsm", "LLNN", (700, 90)), ("trsm", "RUCN", (80, 600)),
                                                ("trsm", "LUTU", (300, 200)), ("trmm", "LLCN", (500, 300)),
                                                ("hemm", "LU", (600, 300)), ("hemm", "RL", (200, 500)),
                                                ("symm", "LL", (400, 300))])
@pytest.mark.parametrize("dtype,method", [("z", eb.METHOD_NATIVE), ("z", eb.METHOD_CRT), ("c", eb.METHOD_AUTO)])
def test_recursion_against_reference(routine, chars, dims, dtype, method):
    rng = np.random.default_rng(hash((routine, chars, dims)) % 2**32)
    npdt = np.complex128 if dtype == "z" else np.complex64
    m, n = dims
    size = m if chars[0] == "L" else n

    def cmat(rows, cols):
        return np.asfortranarray((rng.uniform(-1, 1, (rows, cols)) + 1j * rng.uniform(-1, 1, (rows, cols))).astype(npdt))

    A = cmat(size + 3, size)
    if routine == "trsm":
        sq = A[:size, :size]
        sq *= 1.0 / size
        np.fill_diagonal(sq, (rng.uniform(1, 2, size) * np.exp(1j * rng.uniform(0, 6.28, size))).astype(npdt))
    c = dict(dtype=dtype, routine=routine, chars=chars, dims=list(dims), alpha=0.75 - 0.25j, A=A, B=cmat(m + 1, n))
    if routine in ("hemm", "symm"):
        c["beta"], c["C"] = -0.5 + 1j, cmat(m + 2, n)
    else:
        c["beta"] = None
    (eb.set_dgemm_method if dtype == "z" else eb.set_sgemm_method)(method)
    got = run_ours(c)
    assert eb.last_error()[0] == eb.EB2_OK, eb.last_error()
    c["out"] = _reference(c)
    check(c, got)
