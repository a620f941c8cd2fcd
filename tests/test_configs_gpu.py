"""The benchmark's configurations as parity cases (GPU, through the C ABI).

* plain DGEMM 512^3 (NN, ld = 512, A, B ~ U[-1,1], alpha = 1, beta = 0): the library's
  dgemm_ against Eigen's own dgemm_ built from the reference sources (oracle/_ref), both
  within the product error bound of the exactly rounded result;
* the native-precision sweep: SGEMM and DGEMM, M = N = K in {1024, 2048}, NN / NT / TN,
  alpha = 1.5, beta = 0.5, A, B, C ~ U[-1,1], leading dimensions padded by 8: every method
  within the error bound on a sampled block against the double-double oracle, and the
  emulated methods no less accurate than the native kernels there.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import eigen_b200 as eb
from _helpers import ORACLE_DIR, U32, U64, dd_reference, gemm_error_bound, make_operands

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
REF_BLAS = ORACLE_DIR / "_ref" / "libeigen_ref_blas.so"


@pytest.fixture(autouse=True)
def _defaults():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    eb.load()
    eb.clear_error()
    yield
    eb.set_dgemm_method(eb.METHOD_AUTO)
    eb.set_sgemm_method(eb.METHOD_AUTO)


def _reference_dgemm(A, B, C, m, n, k, alpha, beta, lda, ldb, ldc):
    if not REF_BLAS.exists():
        pytest.skip("oracle/_ref not built (the reference sources were absent)")
    lib = ctypes.CDLL(str(REF_BLAS), mode=ctypes.RTLD_LOCAL)
    i = ctypes.c_int
    Cr = C.copy(order="F")
    lib.dgemm_(b"N", b"N", ctypes.byref(i(m)), ctypes.byref(i(n)), ctypes.byref(i(k)),
               ctypes.byref(ctypes.c_double(alpha)), A.ctypes.data_as(ctypes.c_void_p), ctypes.byref(i(lda)),
               B.ctypes.data_as(ctypes.c_void_p), ctypes.byref(i(ldb)), ctypes.byref(ctypes.c_double(beta)),
               Cr.ctypes.data_as(ctypes.c_void_p), ctypes.byref(i(ldc)))
    return Cr


def test_plain_dgemm_512_against_eigen_dgemm():
    m = n = k = 512
    rng = np.random.default_rng(512)
    A = np.asfortranarray(rng.uniform(-1, 1, (m, k)))
    B = np.asfortranarray(rng.uniform(-1, 1, (k, n)))
    C = np.zeros((m, n), order="F")
    ref = _reference_dgemm(A, B, C, m, n, k, 1.0, 0.0, m, k, m)
    hi, lo = dd_reference("N", "N", m, n, k, 1.0, A, m, B, k, 0.0, C, m)
    bound = gemm_error_bound(A, "N", B, "N", m, n, k, 1.0, 0.0, C, U64)
    assert np.all(np.abs(ref - hi) <= bound)  # the reference itself
    for method in (eb.METHOD_AUTO, eb.METHOD_NATIVE, eb.METHOD_CRT):
        eb.set_dgemm_method(method)
        got = C.copy(order="F")
        eb.dgemm("N", "N", m, n, k, 1.0, A, m, B, k, 0.0, got, m)
        assert eb.last_error()[0] == eb.EB2_OK
        assert np.all(np.abs(got - hi) <= bound), method
        if method == eb.METHOD_CRT:  # as accurate as the reference, or more
            assert np.linalg.norm((got - hi) - lo) <= np.linalg.norm((ref - hi) - lo)


@pytest.mark.parametrize("size", [1024, 2048])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N")])
@pytest.mark.parametrize("dtype", ["d", "s"])
def test_native_precision_sweep(size, ta, tb, dtype):
    m = n = k = size
    npdt = np.float64 if dtype == "d" else np.float32
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, ta, tb, pad=8, seed=size + ord(ta) + 3 * ord(tb),
                                           dtype=npdt)
    rng = np.random.default_rng(size)
    rows = np.sort(rng.choice(m, 40, replace=False))
    cols = np.sort(rng.choice(n, 40, replace=False))
    A64, B64, C64 = (x.astype(np.float64) for x in (A, B, C))
    hi, lo = dd_reference(ta, tb, m, n, k, 1.5, A64, lda, B64, ldb, 0.5, C64, ldc, rows, cols)
    eps = U64 if dtype == "d" else U32
    bound = gemm_error_bound(A64, ta, B64, tb, m, n, k, 1.5, 0.5, C64, eps)[np.ix_(rows, cols)]
    methods = (eb.METHOD_NATIVE, eb.METHOD_CRT, eb.METHOD_EMULATED) if dtype == "d" else (eb.METHOD_NATIVE,
                                                                                          eb.METHOD_EMULATED)
    errs = {}
    for method in methods:
        (eb.set_dgemm_method if dtype == "d" else eb.set_sgemm_method)(method)
        got = C.copy(order="F")
        (eb.dgemm if dtype == "d" else eb.sgemm)(ta, tb, m, n, k, 1.5, A, lda, B, ldb, 0.5, got, ldc)
        assert eb.last_error()[0] == eb.EB2_OK, eb.last_error()
        blk = got[np.ix_(rows, cols)].astype(np.float64)
        assert np.all(np.abs(blk - hi) <= bound), method
        errs[method] = np.linalg.norm((blk - hi) - lo)
        np.testing.assert_array_equal(got[m:, :], C[m:, :])  # padding rows untouched
    # DGEMM: the emulations are at least as accurate as the FP64 kernel; SGEMM: bf16x6 stays
    # within a small factor of FP32 FFMA
    limit = 1.5 if dtype == "d" else 4.0
    for method in methods[1:]:
        assert errs[method] <= limit * errs[eb.METHOD_NATIVE] + 1e-300, errs


def _dev_operand(rows, cols, pad, gen, tdt):
    """Column-major rows x cols matrix with leading dimension rows + pad, entries U[-1,1], on
    the device: a (cols, ld) row-major tensor holds the column-major bytes."""
    ld = rows + pad
    return (torch.rand((cols, ld), dtype=torch.float64, device="cuda", generator=gen) * 2 - 1).to(tdt), ld


def _op_rows(X, trans, idx, k):
    """Rows idx of op(X) (op(X) is len x k) as a host float64 array, from the device tensor."""
    if trans == "N":  # op(X)(i, l) = X[i + l*ld]: element (i, l) is X_t[l, i]
        return X[:k, idx].T.double().cpu().numpy()
    return X[idx, :k].double().cpu().numpy()  # op(X)(i, l) = X[l + i*ld] = X_t[i, l]


@pytest.mark.parametrize("size", [4096, 8192])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N")])
@pytest.mark.parametrize("dtype", ["d", "s"])
def test_native_precision_sweep_large(size, ta, tb, dtype):
    """The sweep's 4096 and 8192 cases with device operands through dgemm_ / sgemm_ (alpha = 1.5,
    beta = 0.5, leading dimensions + 8): each method within the error bound on a sampled 32 x 32
    block against the double-double oracle, the DGEMM emulations at least as accurate as the FP64
    kernel there and split-BF16 SGEMM within 4x of the FP32 FFMA kernel's error."""
    m = n = k = size
    tdt = torch.float64 if dtype == "d" else torch.float32
    gen = torch.Generator(device="cuda")
    gen.manual_seed(size + ord(ta) + 3 * ord(tb))
    A, lda = _dev_operand(*((m, k) if ta == "N" else (k, m)), 8, gen, tdt)
    B, ldb = _dev_operand(*((k, n) if tb == "N" else (n, k)), 8, gen, tdt)
    C0, ldc = _dev_operand(m, n, 8, gen, tdt)
    rng = np.random.default_rng(size)
    rows = np.sort(rng.choice(m, 32, replace=False))
    cols = np.sort(rng.choice(n, 32, replace=False))
    ti = torch.from_numpy(rows).cuda()
    tj = torch.from_numpy(cols).cuda()
    As = np.asfortranarray(_op_rows(A, ta, ti, k))            # 32 x k: rows of op(A)
    Bs = np.asfortranarray(_op_rows(B, "T" if tb == "N" else "N", tj, k).T)  # k x 32: columns of op(B)
    Cs = np.asfortranarray(C0[tj][:, ti].T.double().cpu().numpy())  # C(rows, cols)
    hi, lo = dd_reference("N", "N", 32, 32, k, 1.5, As, 32, Bs, k, 0.5, Cs, 32)
    eps = U64 if dtype == "d" else U32
    bound = gemm_error_bound(As, "N", Bs, "N", 32, 32, k, 1.5, 0.5, Cs, eps)
    methods = (eb.METHOD_NATIVE, eb.METHOD_CRT, eb.METHOD_EMULATED) if dtype == "d" else (eb.METHOD_NATIVE,
                                                                                          eb.METHOD_EMULATED)
    errs = {}
    for method in methods:
        (eb.set_dgemm_method if dtype == "d" else eb.set_sgemm_method)(method)
        C = C0.clone()
        (eb.dgemm if dtype == "d" else eb.sgemm)(ta, tb, m, n, k, 1.5, A, lda, B, ldb, 0.5, C, ldc)
        torch.cuda.synchronize()
        assert eb.last_error()[0] == eb.EB2_OK, eb.last_error()
        blk = C[tj][:, ti].T.double().cpu().numpy()
        assert np.all(np.abs(blk - hi) <= bound), method
        errs[method] = np.linalg.norm((blk - hi) - lo)
        assert torch.equal(C[:, m:], C0[:, m:])  # padding rows of C untouched
        del C
    limit = 1.5 if dtype == "d" else 4.0
    for method in methods[1:]:
        assert errs[method] <= limit * errs[eb.METHOD_NATIVE] + 1e-300, errs
