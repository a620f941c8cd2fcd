"""The other level-3 routines on the GPU, through the C ABI: ?gemmtr_, ?syrk_, ?syr2k_, ?symm_,
?trmm_, ?trsm_ against Eigen's own routines (blas/level3_impl.h:98-754).

* every golden case recorded from the reference (tests/golden/level3_golden.npz: all character
  arguments, sizes from the netlib tester's grid, alpha/beta edge values, NaN in every entry the
  routine must not read): the result within the product error bound of the exact result, as the
  reference's own result is; entries outside the result (the other triangle of C, padding rows)
  bit for bit unchanged; host and device operands;
* sizes that exercise the recursive blocking (triangles split in halves down to 1024 for gemmtr,
  64 for trmm/trsm) against the reference library called on the same inputs, for the FP64
  kernel and the CRT emulation.

Bounds: lam*sqrt(k+2)*u*(|alpha| |X||Y| + |beta| |C|) per entry (the probabilistic bound of
test/product_test_helpers.h:11-40), with k the inner dimension; for trsm the same bound on the
residual op(A) X - alpha B (or X op(A) - alpha B) with |op(A)||X| + |alpha B|.
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
GOLDEN = Path(__file__).resolve().parent / "golden" / "level3_golden.npz"
REF_BLAS = ORACLE_DIR / "_ref" / "libeigen_ref_blas.so"
LAM = 5.0


@pytest.fixture(autouse=True)
def _defaults():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    eb.load()
    eb.clear_error()
    yield
    eb.set_dgemm_method(eb.METHOD_AUTO)
    eb.set_sgemm_method(eb.METHOD_AUTO)


def _load_golden():
    z = np.load(GOLDEN)
    meta = json.loads(bytes(z["meta"]).decode())
    cases = []
    for i, c in enumerate(meta["cases"]):
        c = dict(c)
        for name in ("A", "B", "C"):
            if f"{name}{i}" in z:
                c[name] = z[f"{name}{i}"]
        c["out"] = z[f"out{i}"]
        cases.append(c)
    return cases


_GOLDEN = None


def golden_cases():
    global _GOLDEN
    if _GOLDEN is None:
        _GOLDEN = _load_golden()
    return _GOLDEN


def output_name(routine):
    return "C" if routine in ("gemmtr", "syrk", "syr2k", "symm") else "B"


def arg_list(case, mats):
    """The routine's Fortran argument list for the case, with the matrices `mats`."""
    r, ch, dims, al, be = case["routine"], case["chars"], case["dims"], case["alpha"], case["beta"]
    A, B, C = mats.get("A"), mats.get("B"), mats.get("C")
    ld = {k: case[k].shape[0] for k in ("A", "B", "C") if k in case}
    if r == "gemmtr":
        return [*ch, *dims, al, A, ld["A"], B, ld["B"], be, C, ld["C"]]
    if r == "syrk":
        return [*ch, *dims, al, A, ld["A"], be, C, ld["C"]]
    if r in ("syr2k", "symm"):
        return [*ch, *dims, al, A, ld["A"], B, ld["B"], be, C, ld["C"]]
    return [*ch, *dims, al, A, ld["A"], B, ld["B"]]


def run_ours(case, device=False):
    """Run the case through the library; returns the output array (host copy)."""
    mats = {k: case[k].copy(order="F") for k in ("A", "B", "C") if k in case}
    if not device:
        eb.level3(case["dtype"] + case["routine"], *arg_list(case, mats))
        return mats[output_name(case["routine"])]
    dev = {k: torch.from_numpy(np.ascontiguousarray(v.T)).cuda() for k, v in mats.items()}
    eb.level3(case["dtype"] + case["routine"], *arg_list(case, dev))
    torch.cuda.synchronize()
    return np.asfortranarray(dev[output_name(case["routine"])].cpu().numpy().T)


def _opx(X, tr, rows, cols, dt):
    X = X.astype(dt)
    return X[:cols, :rows].T if tr.upper() != "N" else X[:rows, :cols]


def _tri(A, size, upper, unit, dt):
    T = np.where(np.triu(np.ones((size, size), bool)) if upper else np.tril(np.ones((size, size), bool)),
                 A[:size, :size].astype(dt), 0).astype(dt)
    if unit:
        np.fill_diagonal(T, 1)
    return T


def _sym(A, size, upper, dt):
    T = _tri(A, size, upper, False, dt)
    return T + np.triu(T, 1).T if upper else T + np.tril(T, -1).T


def expected(case, Bin=None, X=None):
    """(value, magnitude, k, region) for the case: the exact result (or, for trsm, the residual
    of X) in extended precision, the magnitude matrix of its error bound, the inner dimension
    and the index region of the output it covers."""
    dt = np.longdouble if case["dtype"] == "d" else np.float64
    r, ch, (d0, d1), al, be = case["routine"], case["chars"].upper(), case["dims"], case["alpha"], case["beta"]
    A = case["A"]

    def beta_term(C, rows, cols):
        if be == 0:
            return 0, 0
        c = C[:rows, :cols].astype(dt)
        return be * c, abs(be) * np.abs(c)

    if r in ("gemmtr", "syrk", "syr2k"):
        n, k = d0, d1
        up = ch[0] == "U"
        if r == "gemmtr":
            X, Y = _opx(A, ch[1], n, k, dt), _opx(case["B"], ch[2], k, n, dt)
            prod, mag = X @ Y, np.abs(X) @ np.abs(Y)
        elif r == "syrk":
            X = _opx(A, "N" if ch[1] == "N" else "T", n, k, dt)
            prod, mag = X @ X.T, np.abs(X) @ np.abs(X).T
        else:
            X = _opx(A, "N" if ch[1] == "N" else "T", n, k, dt)
            Y = _opx(case["B"], "N" if ch[1] == "N" else "T", n, k, dt)
            prod = X @ Y.T + Y @ X.T
            mag = np.abs(X) @ np.abs(Y).T + np.abs(Y) @ np.abs(X).T
        bt, bm = beta_term(case["C"], n, n)
        region = np.triu(np.ones((n, n), bool)) if up else np.tril(np.ones((n, n), bool))
        return al * prod + bt, abs(al) * mag + bm, k, region
    if r == "symm":
        m, n = d0, d1
        left = ch[0] == "L"
        size = m if left else n
        S = _sym(A, size, ch[1] == "U", dt)
        Bm = case["B"][:m, :n].astype(dt)
        prod, mag = (S @ Bm, np.abs(S) @ np.abs(Bm)) if left else (Bm @ S, np.abs(Bm) @ np.abs(S))
        bt, bm = beta_term(case["C"], m, n)
        return al * prod + bt, abs(al) * mag + bm, size, np.ones((m, n), bool)
    m, n = d0, d1
    left = ch[0] == "L"
    size = m if left else n
    T = _tri(A, size, ch[1] == "U", ch[3] == "U", dt)
    opT = T.T if ch[2] != "N" else T
    B0 = (case["B"] if Bin is None else Bin)[:m, :n].astype(dt)
    if r == "trmm":
        prod, mag = (opT @ B0, np.abs(opT) @ np.abs(B0)) if left else (B0 @ opT, np.abs(B0) @ np.abs(opT))
        return al * prod, abs(al) * mag, size, np.ones((m, n), bool)
    Xs = X[:m, :n].astype(dt)
    res = (opT @ Xs if left else Xs @ opT) - al * B0
    mag = (np.abs(opT) @ np.abs(Xs) if left else np.abs(Xs) @ np.abs(opT)) + abs(al) * np.abs(B0)
    return res, mag, size, np.ones((m, n), bool)


def check_case(case, got, eps_scale=1.0):
    """`got` within the bound; everything outside the result untouched; NaN/Inf like the reference."""
    r = case["routine"]
    ref = case["out"]
    inp = case[output_name(r)]
    d0, d1 = case["dims"]
    rows, cols = (d0, d0) if r in ("gemmtr", "syrk", "syr2k") else (d0, d1)
    np.testing.assert_array_equal(got[rows:, :], inp[rows:, :])  # padding rows
    if rows == 0 or cols == 0:
        np.testing.assert_array_equal(got, inp)
        return
    val, mag, k, region = expected(case, X=got if r == "trsm" else None)
    g, rf = got[:rows, :cols], ref[:rows, :cols]
    np.testing.assert_array_equal(g[~region], inp[:rows, :cols][~region])  # the other triangle
    np.testing.assert_array_equal(np.isnan(g), np.isnan(rf))
    np.testing.assert_array_equal(np.isinf(g), np.isinf(rf))
    fin = region & np.isfinite(rf)
    eps = (U64 if case["dtype"] == "d" else U32) * eps_scale
    bound = LAM * np.sqrt(k + 2) * eps * mag.astype(np.float64) + 1e-300
    if r == "trsm":
        assert np.all(np.abs(val.astype(np.float64))[fin] <= bound[fin]), case
        # the reference's solution meets the same residual bound
        rv, rm, _, _ = expected(case, X=ref)
        rb = LAM * np.sqrt(k + 2) * eps * rm.astype(np.float64) + 1e-300
        assert np.all(np.abs(rv.astype(np.float64))[fin] <= rb[fin])
        return
    err = np.abs(g.astype(np.float64) - val.astype(np.float64))
    assert np.all(err[fin] <= bound[fin]), (case, float(np.max(err[fin] / bound[fin])))
    ref_err = np.abs(rf.astype(np.float64) - val.astype(np.float64))
    assert np.all(ref_err[fin] <= bound[fin])  # the bound holds for the reference too


@pytest.mark.parametrize("method", [eb.METHOD_NATIVE, eb.METHOD_CRT])
def test_double_golden(method):
    eb.set_dgemm_method(method)
    n = 0
    for case in golden_cases():
        if case["dtype"] != "d":
            continue
        got = run_ours(case)
        assert eb.last_error()[0] == eb.EB2_OK, (case, eb.last_error())
        check_case(case, got)
        n += 1
    assert n > 600


@pytest.mark.parametrize("method", [eb.METHOD_NATIVE, eb.METHOD_EMULATED])
def test_single_golden(method):
    eb.set_sgemm_method(method)
    for case in golden_cases():
        if case["dtype"] != "s":
            continue
        got = run_ours(case)
        assert eb.last_error()[0] == eb.EB2_OK, (case, eb.last_error())
        check_case(case, got)


@pytest.mark.parametrize("dtype", ["d", "s"])
def test_device_operands_equal_host_operands(dtype):
    """Device (torch) operands are used in place and give the staged call's result bit for bit."""
    for i, case in enumerate(golden_cases()):
        if case["dtype"] != dtype or i % 5:
            continue
        host = run_ours(case)
        dev = run_ours(case, device=True)
        np.testing.assert_array_equal(host, dev)


def test_ilp64_symbols():
    cases = [c for c in golden_cases() if c["dtype"] == "d" and c["dims"] == [9, 5]][:40]
    for case in cases:
        mats = {k: case[k].copy(order="F") for k in ("A", "B", "C") if k in case}
        eb.level3("d" + case["routine"], *arg_list(case, mats), ilp64=True)
        np.testing.assert_array_equal(mats[output_name(case["routine"])], run_ours(case))


# ------------------------------------------------------------------ sizes that recurse
def _ref_lib():
    if not REF_BLAS.exists():
        pytest.skip("oracle/_ref not built (the reference sources were absent)")
    return ctypes.CDLL(str(REF_BLAS), mode=ctypes.RTLD_LOCAL)


def _ref_call(lib, name, values, dtype):
    ctype = ctypes.c_double if dtype == "d" else ctypes.c_float
    out, keep = [], []
    for kind, v in zip(eb.LEVEL3_SIGNATURES[name], values):
        if kind == "c":
            out.append(ctypes.c_char_p(v.encode()))
        elif kind == "a":
            out.append(ctypes.c_void_p(int(v.ctypes.data)))
        else:
            x = ctypes.c_int(v) if kind == "i" else ctype(v)
            keep.append(x)
            out.append(ctypes.cast(ctypes.byref(x), ctypes.c_void_p))
    getattr(lib, dtype + name + "_")(*out)


def _big_case(rng, dtype, routine, chars, dims, alpha, beta):
    npdt = np.float64 if dtype == "d" else np.float32

    def mat(rows, cols, pad=3):
        return np.asfortranarray(rng.uniform(-1, 1, (rows + pad, cols)).astype(npdt))

    c = dict(dtype=dtype, routine=routine, chars=chars, dims=list(dims), alpha=alpha, beta=beta, special=None)
    d0, d1 = dims
    if routine in ("gemmtr", "syrk", "syr2k"):
        n, k = d0, d1
        if routine == "gemmtr":
            c["A"] = mat(*((n, k) if chars[1] == "N" else (k, n)))
            c["B"] = mat(*((k, n) if chars[2] == "N" else (n, k)))
        else:
            c["A"] = mat(*((n, k) if chars[1] == "N" else (k, n)))
            if routine == "syr2k":
                c["B"] = mat(*((n, k) if chars[1] == "N" else (k, n)))
        c["C"] = mat(n, n)
        other = ~(np.triu(np.ones((n, n), bool)) if chars[0] == "U" else np.tril(np.ones((n, n), bool)))
        c["C"][:n, :n][other] = np.nan
    elif routine == "symm":
        size = d0 if chars[0] == "L" else d1
        c["A"], c["B"], c["C"] = mat(size, size), mat(d0, d1), mat(d0, d1)
    else:
        size = d0 if chars[0] == "L" else d1
        A = mat(size, size)
        if routine == "trsm":
            sq = A[:size, :size]
            sq *= 1.0 / size
            np.fill_diagonal(sq, rng.choice([-1.0, 1.0], size) * rng.uniform(1.0, 2.0, size))
        c["A"], c["B"] = A, mat(d0, d1)
    return c


def _run_ref(lib, case):
    mats = {k: case[k].copy(order="F") for k in ("A", "B", "C") if k in case}
    _ref_call(lib, case["routine"], arg_list(case, mats), case["dtype"])
    return mats[output_name(case["routine"])]


BIG = [("gemmtr", "UNN", (1500, 700)), ("gemmtr", "LTN", (1500, 700)), ("gemmtr", "UNT", (2300, 300)),
       ("gemmtr", "LTT", (1100, 257)), ("syrk", "UN", (1500, 500)), ("syrk", "LT", (1300, 600)),
       ("syr2k", "LN", (1100, 300)), ("syr2k", "UT", (1030, 200)), ("symm", "LU", (700, 500)),
       ("symm", "RL", (300, 900))]
TRI = [(r, s + u + t + d, dims) for r in ("trmm", "trsm") for s in "LR" for u in "UL" for t in "NT" for d in "NU"
       for dims in ((300, 200),)] + [("trsm", "LLNN", (700, 200)), ("trmm", "RUTN", (500, 1000)),
                                   ("trmm", "LUNU", (1100, 300)), ("trmm", "RLTN", (200, 1300))]


@pytest.mark.parametrize("routine,chars,dims", BIG + TRI)
@pytest.mark.parametrize("dtype,method", [("d", eb.METHOD_NATIVE), ("d", eb.METHOD_CRT), ("s", eb.METHOD_AUTO)])
def test_recursive_blocking_against_reference(routine, chars, dims, dtype, method):
    lib = _ref_lib()
    rng = np.random.default_rng(hash((routine, chars, dims)) % 2**32)
    case = _big_case(rng, dtype, routine, chars, dims, 0.75 if routine != "trsm" else -1.25,
                     0.5 if routine in ("gemmtr", "syrk", "syr2k", "symm") else 0.0)
    (eb.set_dgemm_method if dtype == "d" else eb.set_sgemm_method)(method)
    got = run_ours(case)
    assert eb.last_error()[0] == eb.EB2_OK, eb.last_error()
    case["out"] = _run_ref(lib, case)
    # the reference's result defines the NaN pattern and untouched entries; the bound is the
    # exact-result bound doubled (both results are within it)
    inp = case[output_name(routine)]
    d0, d1 = dims
    rows, cols = (d0, d0) if routine in ("gemmtr", "syrk", "syr2k") else (d0, d1)
    np.testing.assert_array_equal(got[rows:, :], inp[rows:, :])
    if routine == "trsm":
        val, mag, k, _ = expected(dict(case, A=case["A"]), X=got)
        eps = U64 if dtype == "d" else U32
        bound = LAM * np.sqrt(k + 2) * eps * mag.astype(np.float64)
        assert np.all(np.abs(val.astype(np.float64)) <= bound)
        rel = np.linalg.norm(got[:rows, :cols] - case["out"][:rows, :cols]) / np.linalg.norm(case["out"][:rows, :cols])
        assert rel <= 50 * np.sqrt(k) * eps
        return
    g, rf = got[:rows, :cols].astype(np.float64), case["out"][:rows, :cols].astype(np.float64)
    _, mag, k, region = expected(dict(case, dtype="s"), X=None)  # magnitudes in float64 suffice
    np.testing.assert_array_equal(g[~region], inp[:rows, :cols][~region].astype(np.float64))
    eps = U64 if dtype == "d" else U32
    bound = 2 * LAM * np.sqrt(k + 2) * eps * mag
    assert np.all(np.abs(g - rf)[region] <= bound[region]), float(np.max((np.abs(g - rf) / bound)[region]))


def test_symm_and_trmm_beta_alpha_zero_read_no_operand():
    """alpha == 0: symm leaves beta*C (beta == 0: zeros, NaN in C discarded) without reading A/B."""
    m, n = 70, 40
    A = np.full((m, m), np.nan, order="F")
    B = np.full((m, n), np.nan, order="F")
    C = np.full((m, n), np.nan, order="F")
    eb.level3("dsymm", "L", "U", m, n, 0.0, A, m, B, m, 0.0, C, m)
    assert np.all(C == 0.0)
    C = np.full((m, n), 2.0, order="F")
    eb.level3("dsymm", "R", "L", m, n, 0.0, A[:n], n, B, m, 1.5, C, m)
    assert np.all(C == 3.0)


def test_syrk_k_zero_scales_only_the_triangle():
    n = 50
    C = np.asfortranarray(np.arange(n * n, dtype=np.float64).reshape(n, n))
    C0 = C.copy(order="F")
    a = np.zeros(1)
    eb.level3("dsyrk", "L", "N", n, 0, 1.0, a, n, 2.0, C, n)
    low = np.tril(np.ones((n, n), bool))
    np.testing.assert_array_equal(C[low], 2.0 * C0[low])
    np.testing.assert_array_equal(C[~low], C0[~low])
    eb.level3("dsyrk", "U", "T", n, 0, 1.0, a, 1, 0.0, C, n)
    up = np.triu(np.ones((n, n), bool))
    assert np.all(C[up] == 0.0)
    np.testing.assert_array_equal(C[~up], (2.0 * C0)[~up])


def test_trsm_alpha_applied_after_the_solve():
    """B := alpha * op(A)^-1 B: with alpha == 0 the solve still runs and B is multiplied by 0."""
    m, n = 130, 20
    rng = np.random.default_rng(3)
    A = np.asfortranarray(np.eye(m) * 2.0 + np.tril(rng.uniform(-1, 1, (m, m)) / m, -1))
    B = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
    B[5, 3] = np.inf
    eb.level3("dtrsm", "L", "L", "N", "N", m, n, 0.0, A, m, B, m)
    assert np.isnan(B[5, 3]) and np.all(B[:5, :] == 0.0) and np.all(np.isnan(B[5:, 3]) | (B[5:, 3] == 0.0))


# ------------------------------------------------------------------ the CRT triangle product
@pytest.mark.parametrize("tile_n", [256, 512, 1024])
@pytest.mark.parametrize("n,k,uplo,trans,group", [(700, 300, "L", "N", 0), (1024, 512, "U", "T", 0),
                                                  (1500, 257, "U", "N", 3), (2100, 1000, "L", "T", 2)])
def test_crt_syrk_is_the_triangle_of_the_full_product(tile_n, n, k, uplo, trans, group):
    """dsyrk on the CRT path computes only the tiles meeting the triangle (one split of A serves
    both operands): bit for bit the triangle of the full CRT product of A and a separate copy of
    A, the other triangle untouched."""
    eb.set_dgemm_method(eb.METHOD_CRT)
    eb.set_dgemm_moduli(16)
    eb.set_tile_n(tile_n)
    eb.set_slice_tuning(group, 0)
    try:
        rng = np.random.default_rng(n + k)
        rows, cols = (n, k) if trans == "N" else (k, n)
        A = np.asfortranarray(rng.uniform(-1, 1, (rows + 2, cols)))
        C = np.asfortranarray(rng.uniform(-1, 1, (n + 1, n)))
        up = np.triu(np.ones((n, n), bool)) if uplo == "U" else np.tril(np.ones((n, n), bool))
        C[:n, :n][~up] = np.nan
        got = C.copy(order="F")
        eb.level3("dsyrk", uplo, trans, n, k, 0.75, A, rows + 2, -0.5, got, n + 1)
        assert eb.last_error()[0] == eb.EB2_OK, eb.last_error()
        info = eb.last_call_info()
        assert info["method"] == eb.METHOD_CRT and info["slices"] == 16
        full = C.copy(order="F")
        full[:n, :n][~up] = 0.0
        A2 = A.copy(order="F")  # a distinct operand: the general two-operand path
        ta, tb = ("N", "T") if trans == "N" else ("T", "N")
        eb.dgemm(ta, tb, n, n, k, 0.75, A, rows + 2, A2, rows + 2, -0.5, full, n + 1)
        np.testing.assert_array_equal(got[:n, :n][up], full[:n, :n][up])
        np.testing.assert_array_equal(got[:n, :n][~up], C[:n, :n][~up])
        np.testing.assert_array_equal(got[n:], C[n:])
        # the device entry with one tensor in both roles: bit for bit the two-operand product
        dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
        dC = torch.from_numpy(np.ascontiguousarray(np.where(np.isnan(C), 0.0, C).T)).cuda()
        dC[:n, :n][torch.from_numpy(~up.T).cuda()] = 0.0
        rc = eb.dgemm_device(ta, tb, n, n, k, 0.75, dA, rows + 2, dA, rows + 2, -0.5, dC, n + 1)
        torch.cuda.synchronize()
        assert rc == eb.EB2_OK, eb.last_error()
        np.testing.assert_array_equal(np.asfortranarray(dC.cpu().numpy().T)[:n], full[:n])
    finally:
        eb.set_dgemm_moduli(0)
        eb.set_tile_n(0)
        eb.set_slice_tuning(0, 0)


def test_crt_syrk_nonfinite_input_keeps_the_other_triangle():
    """A NaN in A sends the triangle product to the FP64 kernel (into a workspace, merged into
    the triangle): the other triangle stays untouched, the NaN row and column propagate."""
    eb.set_dgemm_method(eb.METHOD_CRT)
    n, k = 600, 400
    rng = np.random.default_rng(5)
    A = np.asfortranarray(rng.uniform(-1, 1, (n, k)))
    A[17, 3] = np.nan
    C = np.asfortranarray(rng.uniform(-1, 1, (n, n)))
    got = C.copy(order="F")
    eb.level3("dsyrk", "L", "N", n, k, 1.0, A, n, 1.0, got, n)
    assert eb.last_call_info()["nonfinite"] == 1
    low = np.tril(np.ones((n, n), bool))
    np.testing.assert_array_equal(got[~low], C[~low])
    nan_rows = np.isnan(got)
    expect = np.zeros((n, n), bool)
    expect[17, :] = True
    expect[:, 17] = True
    np.testing.assert_array_equal(nan_rows, expect & low)
    want = C + A @ A.T
    fin = low & ~expect
    assert np.max(np.abs(got[fin] - want[fin])) < 1e-12
