"""zgemm_ / cgemm_ on the GPU, through the C ABI, against Eigen's own complex GEMM
(blas/level3_impl.h:12-96 for std::complex, blas/complex_double.cpp / complex_single.cpp).

* every golden case recorded from the reference (tests/golden/complex_golden.npz: all nine
  (transa, transb) pairs with conjugate transposes, sizes from the netlib tester's grid, complex
  alpha/beta including 0 and 1, NaN/Inf in operands that alpha == 0 leaves unread and in a C
  that beta == 0 overwrites): within the product error bound of the reference's result, NaN/Inf
  where it has them, padding rows untouched, for host and device operands and both precisions'
  product methods;
* larger products against the reference library called on the same inputs.

Bound: lam*sqrt(k+2)*u*(|alpha| |op(A)||op(B)| + |beta| |C|) per entry with complex moduli,
lam = 8 (the real bound's 5 with room for the complex multiply's two roundings).
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
GOLDEN = Path(__file__).resolve().parent / "golden" / "complex_golden.npz"
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
            c = dict(c, A=z[f"A{i}"], B=z[f"B{i}"], Cin=z[f"Cin{i}"], Cout=z[f"Cout{i}"])
            c["alpha"], c["beta"] = complex(*c["alpha"]), complex(*c["beta"])
            _CASES.append(c)
    return _CASES


def op(X, t, rows, cols):
    if t.upper() == "N":
        return X[:rows, :cols]
    Y = X[:cols, :rows].T
    return Y.conj() if t.upper() == "C" else Y


def run_ours(c, device=False):
    C = c["Cin"].copy(order="F")
    args = (c["ta"], c["tb"], c["m"], c["n"], c["k"], c["alpha"])
    if not device:
        eb.complex_gemm(c["dtype"], *args, c["A"], c["lda"], c["B"], c["ldb"], c["beta"], C, c["ldc"])
        return C
    dev = [torch.from_numpy(np.ascontiguousarray(x.T)).cuda() for x in (c["A"], c["B"], C)]
    eb.complex_gemm(c["dtype"], *args, dev[0], c["lda"], dev[1], c["ldb"], c["beta"], dev[2], c["ldc"])
    torch.cuda.synchronize()
    return np.asfortranarray(dev[2].cpu().numpy().T)


def check(c, got, ref):
    m, n, k = c["m"], c["n"], c["k"]
    np.testing.assert_array_equal(got[m:, :], c["Cin"][m:, :])  # padding rows
    if m == 0 or n == 0:
        np.testing.assert_array_equal(got, c["Cin"])
        return
    g, r = got[:m, :n], ref[:m, :n]
    for part in (np.real, np.imag):
        np.testing.assert_array_equal(np.isnan(part(g)), np.isnan(part(r)))
        np.testing.assert_array_equal(np.isinf(part(g)), np.isinf(part(r)))
    if c["beta"] == 0 and (k == 0 or c["alpha"] == 0):
        assert np.all(g == 0)
        return
    eps = U64 if c["dtype"] == "z" else U32
    mag = abs(c["beta"]) * np.abs(c["Cin"][:m, :n].astype(np.complex128)) if c["beta"] != 0 else 0.0
    if k and c["alpha"] != 0:
        a = np.abs(op(c["A"], c["ta"], m, k).astype(np.complex128))
        b = np.abs(op(c["B"], c["tb"], k, n).astype(np.complex128))
        mag = mag + abs(c["alpha"]) * (a @ b)
    bound = LAM * np.sqrt(k + 2) * eps * mag + 1e-300
    fin = np.isfinite(r)
    err = np.abs(g.astype(np.complex128) - r.astype(np.complex128))
    assert np.all(err[fin] <= bound[fin]), (c["ta"], c["tb"], m, n, k, float(np.max(err[fin] / bound[fin])))


@pytest.mark.parametrize("dtype,method", [("z", eb.METHOD_NATIVE), ("z", eb.METHOD_CRT), ("c", eb.METHOD_NATIVE),
                                          ("c", eb.METHOD_EMULATED)])
def test_golden_parity(dtype, method):
    (eb.set_dgemm_method if dtype == "z" else eb.set_sgemm_method)(method)
    n = 0
    for c in golden_cases():
        if c["dtype"] != dtype:
            continue
        got = run_ours(c)
        assert eb.last_error()[0] == eb.EB2_OK, (c, eb.last_error())
        check(c, got, c["Cout"])
        n += 1
    assert n > 200


@pytest.mark.parametrize("dtype", ["z", "c"])
def test_device_operands_equal_host_operands(dtype):
    for i, c in enumerate(golden_cases()):
        if c["dtype"] != dtype or i % 4:
            continue
        np.testing.assert_array_equal(run_ours(c), run_ours(c, device=True))


def test_ilp64_symbols():
    for c in [c for c in golden_cases() if c["dtype"] == "z" and c["m"] == 9][:30]:
        C = c["Cin"].copy(order="F")
        eb.complex_gemm("z", c["ta"], c["tb"], c["m"], c["n"], c["k"], c["alpha"], c["A"], c["lda"], c["B"],
                        c["ldb"], c["beta"], C, c["ldc"], ilp64=True)
        np.testing.assert_array_equal(C, run_ours(c))


def _reference(c):
    if not REF_BLAS.exists():
        pytest.skip("oracle/_ref not built (the reference sources were absent)")
    lib = ctypes.CDLL(str(REF_BLAS), mode=ctypes.RTLD_LOCAL)
    real = ctypes.c_double if c["dtype"] == "z" else ctypes.c_float
    i = ctypes.c_int
    C = c["Cin"].copy(order="F")
    al = (real * 2)(c["alpha"].real, c["alpha"].imag)
    be = (real * 2)(c["beta"].real, c["beta"].imag)
    getattr(lib, c["dtype"] + "gemm_")(c["ta"].encode(), c["tb"].encode(), ctypes.byref(i(c["m"])),
                                        ctypes.byref(i(c["n"])), ctypes.byref(i(c["k"])), al,
                                        ctypes.c_void_p(c["A"].ctypes.data), ctypes.byref(i(c["lda"])),
                                        ctypes.c_void_p(c["B"].ctypes.data), ctypes.byref(i(c["ldb"])), be,
                                        ctypes.c_void_p(C.ctypes.data), ctypes.byref(i(c["ldc"])))
    return C


@pytest.mark.parametrize("ta,tb,m,n,k", [("N", "C", 700, 500, 900), ("T", "N", 1000, 1000, 1000),
                                         ("C", "T", 513, 257, 1025), ("N", "N", 2048, 1536, 640)])
@pytest.mark.parametrize("dtype,method", [("z", eb.METHOD_NATIVE), ("z", eb.METHOD_CRT), ("c", eb.METHOD_AUTO)])
def test_larger_products_against_reference(ta, tb, m, n, k, dtype, method):
    rng = np.random.default_rng(m + 3 * n + 7 * k)
    npdt = np.complex128 if dtype == "z" else np.complex64

    def cmat(rows, cols):
        return np.asfortranarray((rng.uniform(-1, 1, (rows, cols)) + 1j * rng.uniform(-1, 1, (rows, cols)))
                                 .astype(npdt))

    ar, ac = (k, m) if ta != "N" else (m, k)
    br, bc = (n, k) if tb != "N" else (k, n)
    c = dict(dtype=dtype, ta=ta, tb=tb, m=m, n=n, k=k, alpha=0.75 - 0.5j, beta=-0.25 + 1j, lda=ar + 3, ldb=br + 1,
             ldc=m + 2)
    c["A"], c["B"], c["Cin"] = cmat(ar + 3, ac), cmat(br + 1, bc), cmat(m + 2, n)
    (eb.set_dgemm_method if dtype == "z" else eb.set_sgemm_method)(method)
    got = run_ours(c)
    assert eb.last_error()[0] == eb.EB2_OK, eb.last_error()
    ref = _reference(c)
    # both results are within the bound of the exact one: their difference within twice it
    eps = U64 if dtype == "z" else U32
    a = np.abs(op(c["A"], ta, m, k).astype(np.complex128))
    b = np.abs(op(c["B"], tb, k, n).astype(np.complex128))
    mag = abs(c["alpha"]) * (a @ b) + abs(c["beta"]) * np.abs(c["Cin"][:m, :n].astype(np.complex128))
    bound = 2 * LAM * np.sqrt(k + 2) * eps * mag
    err = np.abs(got[:m, :n].astype(np.complex128) - ref[:m, :n].astype(np.complex128))
    assert np.all(err <= bound), float(np.max(err / bound))
    np.testing.assert_array_equal(got[m:, :], c["Cin"][m:, :])
