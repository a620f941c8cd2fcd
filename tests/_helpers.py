"""Shared test helpers: the CPU oracle (oracle/liboracle.so) through ctypes, the
golden fixtures, input generators and tolerance formulas.

The oracle is the checker only; nothing here is used by the product library."""
from __future__ import annotations

import ctypes
import json
import subprocess
from functools import lru_cache
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
ORACLE_DIR = ROOT / "oracle"
GOLDEN = Path(__file__).resolve().parent / "golden" / "gemm_golden.npz"
U64 = 2.0 ** -53  # unit roundoff, binary64
U32 = 2.0 ** -24  # unit roundoff, binary32

_vp = ctypes.c_void_p
_l = ctypes.c_long
_d = ctypes.c_double
_c = ctypes.c_char


def _ensure_built(name: str) -> Path:
    p = ORACLE_DIR / name
    if not p.exists():
        subprocess.run(["make", "-C", str(ORACLE_DIR), "all"], check=True, capture_output=True)
    return p


_recorder = None


def load_xerbla_recorder():
    global _recorder
    if _recorder is None:
        _recorder = ctypes.CDLL(str(_ensure_built("librecord_xerbla.so")), mode=ctypes.RTLD_GLOBAL)
        _recorder.record_xerbla_last_name.restype = ctypes.c_char_p
    return _recorder


@lru_cache(maxsize=1)
def oracle():
    lib = ctypes.CDLL(str(_ensure_built("liboracle.so")))
    lib.oracle_gemm_info.argtypes = [_c, _c, _l, _l, _l, _l, _l, _l]
    lib.oracle_dgemm.argtypes = [_c, _c, _l, _l, _l, _d, _vp, _l, _vp, _l, _d, _vp, _l]
    lib.oracle_sgemm.argtypes = [_c, _c, _l, _l, _l, ctypes.c_float, _vp, _l, _vp, _l, ctypes.c_float, _vp, _l]
    lib.oracle_dgemm_dd.argtypes = [_c, _c, _l, _l, _l, _d, _vp, _l, _vp, _l, _d, _vp, _l, _vp, _l, _vp, _l, _vp, _vp]
    lib.oracle_abs_product_fro.argtypes = [_c, _c, _l, _vp, _l, _vp, _l, _vp, _l, _vp, _l]
    lib.oracle_abs_product_fro.restype = _d
    lib.oracle_dgemm_test_ratio.argtypes = [_c, _c, _l, _l, _l, _d, _vp, _l, _vp, _l, _d, _vp, _l, _vp, _l, _d]
    lib.oracle_dgemm_test_ratio.restype = _d
    lib.oracle_sgemm_test_ratio.argtypes = [_c, _c, _l, _l, _l, ctypes.c_float, _vp, _l, _vp, _l, ctypes.c_float,
                                            _vp, _l, _vp, _l, _d]
    lib.oracle_sgemm_test_ratio.restype = _d
    lib.oracle_ozaki_split.argtypes = [_vp, _l, _l, _l, _l, ctypes.c_int, _vp, _l, _l, _vp]
    lib.oracle_ozaki_dgemm.argtypes = [_c, _c, _l, _l, _l, _d, _vp, _l, _vp, _l, _d, _vp, _l, ctypes.c_int]
    return lib


@lru_cache(maxsize=1)
def crt_model():
    """The exact CPU model of the CRT-form emulated DGEMM (oracle/ozaki2.py)."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("oracle_ozaki2", ORACLE_DIR / "ozaki2.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def P(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(_vp)


def ch(x: str) -> bytes:
    return x.encode()


# ---------------------------------------------------------------- golden fixtures
@lru_cache(maxsize=1)
def golden():
    z = np.load(GOLDEN)
    meta = json.loads(bytes(z["meta"]))
    cases = []
    for i, m in enumerate(meta["cases"]):
        cases.append(dict(m, A=z[f"A{i}"], B=z[f"B{i}"], Cin=z[f"Cin{i}"], Cout=z[f"Cout{i}"]))
    return cases, meta["errors"]


# ---------------------------------------------------------------- inputs
def op_shape(trans: str, rows: int, cols: int) -> tuple[int, int]:
    """Storage shape of X such that op(X) is rows x cols."""
    return (cols, rows) if trans.upper() != "N" else (rows, cols)


def make_operands(m, n, k, ta="N", tb="N", pad=0, r=0, seed=0, dtype=np.float64):
    """Column-major A, B, C with entries u*2^e, u ~ U[-1,1], e ~ U{-r..r}; padded ld."""
    rng = np.random.default_rng(seed)

    def mat(rows, cols):
        ld = max(1, rows + pad)
        x = rng.uniform(-1, 1, (ld, max(cols, 1)))
        if r:
            x *= 2.0 ** rng.integers(-r, r + 1, x.shape)
        return np.asfortranarray(x.astype(dtype)), ld

    A, lda = mat(*op_shape(ta, m, k))
    B, ldb = mat(*op_shape(tb, k, n))
    C, ldc = mat(m, n)
    return A, lda, B, ldb, C, ldc


def op(X, trans, rows, cols):
    """op(X) as a dense rows x cols array."""
    return X[:cols, :rows].T if trans.upper() != "N" else X[:rows, :cols]


def gemm_error_bound(A, ta, B, tb, m, n, k, alpha, beta, Cin, eps, lam=5.0):
    """Per-element bound lam*sqrt(k+2)*eps*(|alpha| |opA||opB| + |beta| |C|) + tiny, after
    the probabilistic bound of test/product_test_helpers.h:11-40 (Higham & Mary 2019)."""
    a = np.abs(op(A, ta, m, k).astype(np.float64))
    b = np.abs(op(B, tb, k, n).astype(np.float64))
    g = abs(alpha) * (a @ b)
    if beta != 0:
        g = g + abs(beta) * np.abs(Cin[:m, :n].astype(np.float64))
    g = np.nan_to_num(g, nan=np.inf, posinf=np.inf)
    return lam * np.sqrt(k + 2) * eps * g + 1e-300


def dd_reference(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, rows=None, cols=None):
    """alpha*op(A)op(B) + beta*C in double-double on a sub-block (hi + lo)."""
    lib = oracle()
    rows = np.arange(m, dtype=np.int64) if rows is None else np.asarray(rows, dtype=np.int64)
    cols = np.arange(n, dtype=np.int64) if cols is None else np.asarray(cols, dtype=np.int64)
    hi = np.zeros((len(rows), len(cols)), order="F")
    lo = np.zeros_like(hi)
    lib.oracle_dgemm_dd(ch(ta), ch(tb), m, n, k, alpha, P(A), lda, P(B), ldb, beta, P(C), ldc, P(rows), len(rows),
                        P(cols), len(cols), P(hi), P(lo))
    return hi, lo


def rel_error_vs_dd(Cout, hi, lo, rows=None, cols=None, Cref_norm=None):
    """||C - C_dd||_F / ||C_dd||_F on the sampled block."""
    sub = Cout if rows is None else Cout[np.ix_(rows, cols)]
    err = np.linalg.norm((sub - hi) - lo)
    nrm = np.linalg.norm(hi) if Cref_norm is None else Cref_norm
    return err / nrm if nrm else err


def check_against_reference(case, C, eps_scale=1.0):
    """Bit-exact where the reference's result is exact (alpha == 0, k == 0, m or n == 0),
    NaN/Inf pattern identical, otherwise within the product error bound."""
    ref = case["Cout"]
    m, n, k = case["m"], case["n"], case["k"]
    if m == 0 or n == 0:
        np.testing.assert_array_equal(C, ref)
        return
    c, r = C[:m, :n], ref[:m, :n]
    np.testing.assert_array_equal(np.isnan(c), np.isnan(r))
    np.testing.assert_array_equal(np.isinf(c), np.isinf(r))
    fin = np.isfinite(r)
    if k == 0 or case["alpha"] == 0.0:
        np.testing.assert_array_equal(c[fin], r[fin])
        return
    eps = (U64 if case["dtype"] == "d" else U32) * eps_scale
    bound = gemm_error_bound(case["A"], case["ta"], case["B"], case["tb"], m, n, k, case["alpha"], case["beta"],
                             case["Cin"], eps)
    assert np.all(np.abs(c - r)[fin] <= bound[fin])
    # padding rows of C (ldc > m) are never touched
    np.testing.assert_array_equal(C[m:, :], case["Cin"][m:, :])
