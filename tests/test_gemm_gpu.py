"""Parity of the B200 product path with the reference, through the C ABI (GPU).

* every golden case of Eigen's own sgemm_/dgemm_ (tests/golden), host and device
  buffers, native and emulated methods;
* the emulated DGEMM bit for bit against the oracle's operation-for-operation model;
* accuracy of the emulated DGEMM against a double-double oracle versus the native
  FP64 kernel, with the a-posteriori slice escalation;
* BLAS edge semantics: alpha == 0, beta == 0, NaN/Inf, k == 0, ILP64.
"""
from __future__ import annotations

import numpy as np
import pytest

import eigen_b200 as eb
from _helpers import (P, U64, ch, check_against_reference, dd_reference, golden, make_operands, oracle,
                      rel_error_vs_dd)

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(autouse=True)
def _defaults():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    eb.load()
    eb.set_dgemm_method(eb.METHOD_AUTO)
    eb.set_sgemm_method(eb.METHOD_AUTO)
    eb.set_dgemm_slices(0)
    eb.set_dgemm_tolerance(U64)
    eb.set_tile_n(0)
    eb.set_sgemm_pieces(3)
    eb.clear_error()
    yield
    eb.set_dgemm_method(eb.METHOD_AUTO)
    eb.set_sgemm_method(eb.METHOD_AUTO)
    eb.set_dgemm_slices(0)
    eb.set_dgemm_tolerance(U64)
    eb.set_tile_n(0)


def _call(case, C, device=False):
    f = eb.dgemm if case["dtype"] == "d" else eb.sgemm
    if not device:
        f(case["ta"], case["tb"], case["m"], case["n"], case["k"], case["alpha"], case["A"], case["lda"], case["B"],
          case["ldb"], case["beta"], C, case["ldc"])
        return C
    tA = torch.from_numpy(np.asfortranarray(case["A"]).T.copy()).cuda()  # row-major of A^T == column-major A
    tB = torch.from_numpy(np.asfortranarray(case["B"]).T.copy()).cuda()
    tC = torch.from_numpy(np.asfortranarray(C).T.copy()).cuda()
    f(case["ta"], case["tb"], case["m"], case["n"], case["k"], case["alpha"], tA, case["lda"], tB, case["ldb"],
      case["beta"], tC, case["ldc"])
    torch.cuda.synchronize()
    return np.asfortranarray(tC.cpu().numpy().T)


@pytest.mark.parametrize("method", [eb.METHOD_NATIVE, eb.METHOD_EMULATED])
@pytest.mark.parametrize("device", [False, True])
def test_dgemm_golden_parity(method, device):
    eb.set_dgemm_method(method)
    cases, _ = golden()
    n = 0
    for case in cases:
        if case["dtype"] != "d":
            continue
        C = _call(case, case["Cin"].copy(order="F"), device)
        check_against_reference(case, C)
        assert eb.last_error()[0] == eb.EB2_OK, eb.last_error()
        n += 1
    assert n > 300


@pytest.mark.parametrize("device", [False, True])
def test_sgemm_golden_parity(device):
    eb.set_sgemm_method(eb.METHOD_NATIVE)
    cases, _ = golden()
    for case in cases:
        if case["dtype"] != "s":
            continue
        C = _call(case, case["Cin"].copy(order="F"), device)
        check_against_reference(case, C)


SHAPES = [("N", "N", 130, 300, 257), ("T", "N", 64, 64, 1000), ("N", "T", 333, 129, 64), ("T", "T", 5, 517, 3),
          ("N", "N", 1, 1, 1), ("C", "N", 256, 256, 128), ("N", "N", 129, 1, 777)]


@pytest.mark.parametrize("ta,tb,m,n,k", SHAPES)
@pytest.mark.parametrize("s,tile_n,beta", [(3, 128, 0.0), (8, 256, 0.0), (8, 128, 0.5), (5, 256, -1.25),
                                          (8, 512, 0.0), (4, 512, 0.75)])
def test_emulated_bit_exact_vs_oracle_model(ta, tb, m, n, k, s, tile_n, beta):
    """Digit split, INT8 digit products and FP64 recombination equal the oracle's
    model (oracle_ozaki_dgemm) bit for bit."""
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, ta, tb, pad=3, r=4, seed=m + n + k + s)
    eb.set_dgemm_method(eb.METHOD_EMULATED)
    eb.set_dgemm_slices(s)
    eb.set_dgemm_tolerance(1.0)  # no escalation: exactly s slices
    eb.set_tile_n(tile_n)
    Cg = C.copy(order="F")
    eb.dgemm(ta, tb, m, n, k, 1.5, A, lda, B, ldb, beta, Cg, ldc)
    info = eb.last_call_info()
    assert info["slices"] == s and info["tile_n"] == tile_n and info["escalations"] == 0
    Co = C.copy(order="F")
    oracle().oracle_ozaki_dgemm(ch(ta), ch(tb), m, n, k, 1.5, P(A), lda, P(B), ldb, beta, P(Co), ldc, s)
    np.testing.assert_array_equal(Cg, Co)


@pytest.mark.parametrize("r", [0, 8, 32])
def test_emulated_accuracy_no_worse_than_native(r):
    """Normwise error against a double-double oracle on a sampled block: the emulated
    DGEMM (slices chosen + a-posteriori escalation) is no worse than the native FP64
    kernel, and within its own target."""
    m = n = k = 1024
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, "N", "N", pad=8, r=r, seed=100 + r)
    rng = np.random.default_rng(r)
    rows = np.sort(rng.choice(m, 48, replace=False))
    cols = np.sort(rng.choice(n, 48, replace=False))
    hi, lo = dd_reference("N", "N", m, n, k, 1.0, A, lda, B, ldb, 0.0, None, ldc, rows, cols)
    errs = {}
    for method in (eb.METHOD_NATIVE, eb.METHOD_EMULATED):
        eb.set_dgemm_method(method)
        Cg = C.copy(order="F")
        eb.dgemm("N", "N", m, n, k, 1.0, A, lda, B, ldb, 0.0, Cg, ldc)
        errs[method] = rel_error_vs_dd(Cg, hi, lo, rows, cols)
        if method == eb.METHOD_EMULATED:
            info = eb.last_call_info()
            assert 0 <= info["err_estimate"] <= U64
            assert info["slices"] >= 8
    assert errs[eb.METHOD_EMULATED] <= max(errs[eb.METHOD_NATIVE], 2 * U64), errs
    assert errs[eb.METHOD_NATIVE] < 50 * U64, errs


def test_escalation_adds_slices_for_wide_exponent_range():
    m = n = 256
    k = 2048
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, "N", "N", r=32, seed=9)
    eb.set_dgemm_method(eb.METHOD_EMULATED)
    eb.set_dgemm_slices(6)
    Cg = C.copy(order="F")
    eb.dgemm("N", "N", m, n, k, 1.0, A, lda, B, ldb, 0.0, Cg, ldc)
    info = eb.last_call_info()
    assert info["escalations"] >= 2 and info["slices"] == 6 + info["escalations"]
    assert info["err_estimate"] <= U64
    hi, lo = dd_reference("N", "N", m, n, k, 1.0, A, lda, B, ldb, 0.0, None, ldc)
    assert rel_error_vs_dd(Cg, hi, lo) < 4 * U64


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
@pytest.mark.parametrize("method", [eb.METHOD_NATIVE, eb.METHOD_EMULATED])
def test_dgemm_test_ratio(ta, tb, method):
    """The netlib Level-3 check (restated DMMCH, threshold 16) on odd shapes."""
    m, n, k = 261, 135, 300
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, ta, tb, pad=5, seed=17)
    eb.set_dgemm_method(method)
    Cg = C.copy(order="F")
    eb.dgemm(ta, tb, m, n, k, 0.7, A, lda, B, ldb, 1.3, Cg, ldc)
    ratio = oracle().oracle_dgemm_test_ratio(ch(ta), ch(tb), m, n, k, 0.7, P(A), lda, P(B), ldb, 1.3, P(C), ldc,
                                             P(Cg), ldc, U64)
    assert ratio < 16.0
    np.testing.assert_array_equal(Cg[m:, :], C[m:, :])  # rows past m untouched


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
@pytest.mark.parametrize("method", [eb.METHOD_NATIVE, eb.METHOD_EMULATED])
def test_sgemm_test_ratio(ta, tb, method):
    eb.set_sgemm_method(method)
    m, n, k = 261, 135, 300
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, ta, tb, pad=5, seed=19, dtype=np.float32)
    Cg = C.copy(order="F")
    eb.sgemm(ta, tb, m, n, k, 0.7, A, lda, B, ldb, 1.3, Cg, ldc)
    ratio = oracle().oracle_sgemm_test_ratio(ch(ta), ch(tb), m, n, k, 0.7, P(A), lda, P(B), ldb, 1.3, P(C), ldc,
                                             P(Cg), ldc, 2.0 ** -24)
    assert ratio < 16.0


@pytest.mark.parametrize("method", [eb.METHOD_NATIVE, eb.METHOD_EMULATED])
def test_nonfinite_inputs_follow_ieee(method):
    m, n, k = 70, 40, 90
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, "N", "N", seed=23)
    A[3, 5] = np.nan
    B[7, 2] = np.inf
    eb.set_dgemm_method(method)
    Cg = C.copy(order="F")
    eb.dgemm("N", "N", m, n, k, 1.0, A, lda, B, ldb, 0.0, Cg, ldc)
    Co = C.copy(order="F")
    oracle().oracle_dgemm(b"N", b"N", m, n, k, 1.0, P(A), lda, P(B), ldb, 0.0, P(Co), ldc)
    np.testing.assert_array_equal(np.isnan(Cg), np.isnan(Co))
    np.testing.assert_array_equal(np.isinf(Cg), np.isinf(Co))
    if method == eb.METHOD_EMULATED:
        assert eb.last_call_info()["nonfinite"] == 1


@pytest.mark.parametrize("method", [eb.METHOD_NATIVE, eb.METHOD_EMULATED])
def test_alpha_zero_reads_neither_a_nor_b(method):
    """alpha == 0: C = beta*C exactly, even with NaN/Inf in A and B
    (Eigen/src/Core/products/GeneralMatrixMatrix.h:130, test/product_extra.cpp:665-728)."""
    m, n, k = 33, 17, 9
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, "N", "N", seed=29)
    A[:] = np.nan
    B[:] = np.inf
    eb.set_dgemm_method(method)
    for beta in (0.0, 1.0, 1.3):
        Cg = C.copy(order="F")
        eb.dgemm("N", "N", m, n, k, 0.0, A, lda, B, ldb, beta, Cg, ldc)
        expect = np.zeros_like(C) if beta == 0 else C * beta
        np.testing.assert_array_equal(Cg[:m, :n], expect[:m, :n])


def test_beta_zero_discards_nan_in_c():
    m, n, k = 20, 20, 20
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, "N", "N", seed=31)
    C[:] = np.nan
    for method in (eb.METHOD_NATIVE, eb.METHOD_EMULATED):
        eb.set_dgemm_method(method)
        Cg = C.copy(order="F")
        eb.dgemm("N", "N", m, n, k, 1.0, A, lda, B, ldb, 0.0, Cg, ldc)
        assert np.isfinite(Cg[:m, :n]).all()


def test_k_zero_scales_c():
    C = np.asfortranarray(np.arange(12.0).reshape(3, 4))
    Cg = C.copy(order="F")
    eb.dgemm("N", "N", 3, 4, 0, 1.0, np.zeros(1), 3, np.zeros(1), 1, 2.0, Cg, 3)
    np.testing.assert_array_equal(Cg, 2 * C)


def test_ilp64_entry_points():
    m, n, k = 50, 60, 70
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, "T", "N", pad=2, seed=37)
    C1 = C.copy(order="F")
    C2 = C.copy(order="F")
    eb.dgemm("T", "N", m, n, k, 1.0, A, lda, B, ldb, 0.5, C1, ldc)
    eb.dgemm("T", "N", m, n, k, 1.0, A, lda, B, ldb, 0.5, C2, ldc, ilp64=True)
    np.testing.assert_array_equal(C1, C2)


def test_device_entry_on_a_torch_stream():
    m, n, k = 512, 384, 640
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, "N", "N", seed=41)
    s = torch.cuda.Stream()
    tA = torch.from_numpy(A.T.copy()).cuda()
    tB = torch.from_numpy(B.T.copy()).cuda()
    tC = torch.from_numpy(C.T.copy()).cuda()
    torch.cuda.synchronize()
    eb.set_dgemm_method(eb.METHOD_CRT)  # the emulated product's accuracy, whatever the picker would choose
    try:
        rc = eb.dgemm_device("N", "N", m, n, k, 1.0, tA, lda, tB, ldb, 0.0, tC, ldc, stream=s.cuda_stream,
                             check_accuracy=False)
    finally:
        eb.set_dgemm_method(eb.METHOD_AUTO)
    assert rc == eb.EB2_OK
    s.synchronize()
    Cg = np.asfortranarray(tC.cpu().numpy().T)
    hi, lo = dd_reference("N", "N", m, n, k, 1.0, A, lda, B, ldb, 0.0, None, ldc)
    assert rel_error_vs_dd(Cg[:m, :n], hi, lo) < 4 * U64


# ---------------------------------------------------------------- split-BF16 SGEMM
@pytest.mark.parametrize("device", [False, True])
def test_sgemm_emulated_golden_parity(device):
    """bf16x6 (default) meets the FP32 product bound on every golden case."""
    eb.set_sgemm_method(eb.METHOD_EMULATED)
    eb.set_sgemm_pieces(3)
    cases, _ = golden()
    for case in cases:
        if case["dtype"] != "s":
            continue
        C = _call(case, case["Cin"].copy(order="F"), device)
        check_against_reference(case, C)


def _sgemm_rel_err(m, n, k, ta, tb, seed, r=0):
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, ta, tb, pad=3, r=r, seed=seed, dtype=np.float32)
    Cg = C.copy(order="F")
    eb.sgemm(ta, tb, m, n, k, 1.0, A, lda, B, ldb, 0.0, Cg, ldc)
    A64, B64 = A.astype(np.float64), B.astype(np.float64)
    hi, lo = dd_reference(ta, tb, m, n, k, 1.0, A64, lda, B64, ldb, 0.0, None, ldc)
    return rel_error_vs_dd(Cg[:m, :n].astype(np.float64), hi, lo)


@pytest.mark.parametrize("ta,tb,m,n,k", [("N", "N", 640, 384, 1024), ("T", "N", 300, 517, 700),
                                         ("N", "T", 129, 1, 2000), ("T", "T", 257, 260, 64)])
def test_sgemm_split_bf16_accuracy(ta, tb, m, n, k):
    """bf16x6 is about as accurate as the native FP32 kernel (within 4x); bf16x3 loses
    about 8 bits (relative error below 2^-15)."""
    eb.set_sgemm_method(eb.METHOD_NATIVE)
    e_nat = _sgemm_rel_err(m, n, k, ta, tb, seed=5)
    eb.set_sgemm_method(eb.METHOD_EMULATED)
    eb.set_sgemm_pieces(3)
    e6 = _sgemm_rel_err(m, n, k, ta, tb, seed=5)
    info = eb.last_call_info()
    assert info["method"] == eb.METHOD_EMULATED and info["slices"] == 6
    eb.set_sgemm_pieces(2)
    e3 = _sgemm_rel_err(m, n, k, ta, tb, seed=5)
    assert eb.last_call_info()["slices"] == 3
    eb.set_sgemm_pieces(3)
    # FP32 accumulation inside the tensor core is not the FFMA kernel's sequential
    # round-to-nearest chain; both stay far inside the lam*sqrt(k)*eps product bound
    assert e6 <= max(4 * e_nat, 2.0 ** -19), (e6, e_nat)
    assert e3 < 2.0 ** -15, e3


@pytest.mark.parametrize("tile_n", [128, 256, 512])
def test_sgemm_split_bf16_tile_configs(tile_n):
    """Every tile configuration (one CTA 128x128 / 128x256, CTA pair 256x256) gives the
    same FP32-level accuracy on odd shapes."""
    eb.set_sgemm_method(eb.METHOD_EMULATED)
    eb.set_tile_n(tile_n)
    e = _sgemm_rel_err(300, 517, 700, "T", "N", seed=7)
    assert eb.last_call_info()["tile_n"] == tile_n
    assert e < 2.0 ** -19, e


def test_sgemm_emulated_nonfinite_falls_back():
    m, n, k = 70, 40, 90
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, "N", "N", seed=43, dtype=np.float32)
    A[3, 5] = np.nan
    B[7, 2] = np.inf
    eb.set_sgemm_method(eb.METHOD_EMULATED)
    Cg = C.copy(order="F")
    eb.sgemm("N", "N", m, n, k, 1.0, A, lda, B, ldb, 0.0, Cg, ldc)
    assert eb.last_call_info()["nonfinite"] == 1
    Co = C.copy(order="F")
    oracle().oracle_sgemm(b"N", b"N", m, n, k, 1.0, P(A), lda, P(B), ldb, 0.0, P(Co), ldc)
    np.testing.assert_array_equal(np.isnan(Cg), np.isnan(Co))
    np.testing.assert_array_equal(np.isinf(Cg), np.isinf(Co))


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
@pytest.mark.parametrize("m,n,k", [(130, 258, 37), (1026, 514, 300), (8, 1030, 17)])
def test_native_copy_width_keeps_bits(ta, tb, m, n, k):
    """The FP64 kernel copies 16-byte pairs when an operand is 16-byte aligned with an even
    leading dimension and single elements otherwise (ragged edges zero-filled either way): the
    same product through both paths, and across the grouped tile raster, is bit-identical and
    within the FP64 error bound of a float128-free double-double check."""
    eb.set_dgemm_method(eb.METHOD_NATIVE)
    rng = np.random.default_rng(m + n + k)
    rows_a, cols_a = (m, k) if ta == "N" else (k, m)
    rows_b, cols_b = (k, n) if tb == "N" else (n, k)
    A = rng.uniform(-1, 1, (rows_a, cols_a))
    B = rng.uniform(-1, 1, (rows_b, cols_b))
    out = {}
    for pad in (0, 1):  # leading dimension rows (even here) or rows + 1 (odd)
        lda, ldb = rows_a + pad, rows_b + pad
        tA = torch.zeros((cols_a, lda), dtype=torch.float64, device="cuda")
        tB = torch.zeros((cols_b, ldb), dtype=torch.float64, device="cuda")
        tA[:, :rows_a] = torch.from_numpy(A.T.copy()).cuda()
        tB[:, :rows_b] = torch.from_numpy(B.T.copy()).cuda()
        tC = torch.zeros((n, m), dtype=torch.float64, device="cuda")
        rc = eb.dgemm_device(ta, tb, m, n, k, 1.0, tA, lda, tB, ldb, 0.0, tC, m)
        torch.cuda.synchronize()
        assert rc == eb.EB2_OK, eb.last_error()
        out[pad] = tC.cpu().numpy().T.copy()
    np.testing.assert_array_equal(out[0], out[1])
    opA = A if ta == "N" else A.T
    opB = B if tb == "N" else B.T
    want = opA @ opB
    bound = 2 * k * U64 * (np.abs(opA) @ np.abs(opB)) + 1e-300
    assert np.all(np.abs(out[0] - want) <= bound)
