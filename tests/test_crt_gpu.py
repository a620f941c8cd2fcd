"""The CRT-form emulated DGEMM (Ozaki scheme II) through the C ABI (GPU).

* bit for bit against the exact CPU model (oracle/ozaki2.py): norm bounds, scaling,
  truncation, exact integer product, one rounding, alpha/beta;
* the K > 1023 x 128 split of the INT32 accumulation (residues added mod p);
* accuracy against a double-double oracle versus the native FP64 kernel;
* the a-posteriori check adding moduli, with beta == 0 and beta != 0;
* zero rows, NaN/Inf inputs, extreme exponents, host and device entry points.
"""
from __future__ import annotations

import numpy as np
import pytest

import eigen_b200 as eb
from _helpers import U64, crt_model, dd_reference, make_operands, op, rel_error_vs_dd

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(autouse=True)
def _defaults():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    eb.load()
    eb.set_dgemm_method(eb.METHOD_CRT)
    # the count the models below use; the check still adds moduli (a picker would otherwise
    # predict a count from the accuracy target)
    eb.set_dgemm_moduli(16)
    eb.set_dgemm_tolerance(U64)
    eb.set_tile_n(0)
    eb.clear_error()
    yield
    eb.set_dgemm_method(eb.METHOD_AUTO)
    eb.set_dgemm_moduli(0)
    eb.set_dgemm_tolerance(U64)
    eb.set_tile_n(0)


def _model(A, ta, B, tb, m, n, k, alpha, beta, C, moduli):
    out = C.copy(order="F")
    out[:m, :n] = crt_model().crt_dgemm(op(A, ta, m, k), op(B, tb, k, n), alpha, beta, C[:m, :n], moduli)[0]
    return out


def _device_call(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, check):
    dev = [torch.from_numpy(np.asfortranarray(x).T.copy()).cuda() for x in (A, B, C)]
    rc = eb.dgemm_device(ta, tb, m, n, k, alpha, dev[0], lda, dev[1], ldb, beta, dev[2], ldc, check_accuracy=check)
    torch.cuda.synchronize()
    return rc, np.asfortranarray(dev[2].cpu().numpy().T)


SHAPES = [("N", "N", 130, 300, 257), ("T", "N", 64, 64, 1000), ("N", "T", 333, 129, 64), ("T", "T", 5, 517, 3),
          ("N", "N", 1, 1, 1), ("C", "N", 256, 256, 128), ("N", "N", 129, 1, 777)]


@pytest.mark.parametrize("ta,tb,m,n,k", SHAPES)
@pytest.mark.parametrize("moduli,tile_n,beta", [(16, 256, 0.0), (16, 512, 0.5), (20, 256, -1.25), (8, 512, 0.0),
                                                (18, 256, 0.75), (11, 256, 0.25), (15, 512, 0.0), (16, 1024, 0.0),
                                                (12, 1024, 0.5)])
def test_crt_bit_exact_vs_oracle_model(ta, tb, m, n, k, moduli, tile_n, beta):
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, ta, tb, pad=3, r=4, seed=m + n + k + moduli)
    eb.set_dgemm_moduli(moduli)
    eb.set_dgemm_tolerance(1.0)  # no escalation: exactly `moduli` moduli
    eb.set_tile_n(tile_n)
    Cg = C.copy(order="F")
    eb.dgemm(ta, tb, m, n, k, 1.5, A, lda, B, ldb, beta, Cg, ldc)
    info = eb.last_call_info()
    assert info["method"] == eb.METHOD_CRT and info["slices"] == moduli and info["tile_n"] == tile_n
    assert info["escalations"] == 0 and eb.last_error()[0] == eb.EB2_OK
    np.testing.assert_array_equal(Cg, _model(A, ta, B, tb, m, n, k, 1.5, beta, C, moduli))


@pytest.mark.parametrize("r", [60, 300])
def test_crt_bit_exact_wide_exponents(r):
    """Entries u*2^e with |e| <= r: row scales far apart, products near under/overflow of
    the partial terms; no accuracy check (the estimate is not the subject)."""
    m, n, k = 70, 90, 150
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, "N", "T", pad=1, r=r, seed=r)
    for beta in (0.0, 0.25):
        rc, Cg = _device_call("N", "T", m, n, k, -0.75, A, lda, B, ldb, beta, C, ldc, check=False)
        assert rc == eb.EB2_OK
        np.testing.assert_array_equal(Cg, _model(A, "N", B, "T", m, n, k, -0.75, beta, C, 16))


def test_crt_subnormal_and_huge_rows():
    """Rows whose maximum is subnormal or near the top of the range, and zero rows."""
    m, n, k = 40, 33, 64
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, seed=5)
    A[0, :k] *= 2.0 ** -1060          # subnormal row of op(A)
    A[1, :k] *= 2.0 ** 900            # huge row
    A[2, :k] = 0.0                    # zero row
    B[:k, 3] = 0.0                    # zero column of op(B)
    B[:k, 4] *= 2.0 ** -1000
    B[:k, 5] *= 2.0 ** 100            # with the huge row: products near 2^1000
    rc, Cg = _device_call("N", "N", m, n, k, 1.0, A, lda, B, ldb, 0.0, C, ldc, check=False)
    assert rc == eb.EB2_OK
    np.testing.assert_array_equal(Cg, _model(A, "N", B, "N", m, n, k, 1.0, 0.0, C, 16))
    assert np.all(Cg[2, :n] == 0.0) and np.all(Cg[:m, 3] == 0.0)


def _rounding_operands(m, n, rng):
    """op(A) (m x 4) and op(B) (4 x n) with C_ij = y_i x_j + z_i w_j exactly: the first two
    products cancel (1 - 1), y_i = 2^-a_i (1 + 2^-c_i) and x_j = 2^-f_j (1 + 2^-d_j), so C'
    has its top bit where the row and column scales put it and its lowest bit c_i + d_j below
    that: c_i + d_j = 53 is a rounding tie (to even unless c_i or d_j is 52); the lone bit
    z_i w_j below it, in half of the rows, makes it a sticky bit instead.  The column
    exponents f_j spread |C'| over every magnitude window of the rounding, zero rows included."""
    c = rng.integers(1, 53, size=m)
    y = 2.0 ** -rng.integers(0, 3, size=m) * (1 + 2.0 ** -c)
    y[rng.random(m) < 0.05] = 0.0
    z = np.where(rng.random(m) < 0.5, 2.0 ** -rng.integers(56, 60, size=m), 0.0)
    d = rng.integers(1, 53, size=n)
    f = np.array([rng.integers(0, 59 - dj) for dj in d])
    x = 2.0 ** -f * (1 + 2.0 ** -d)
    w = 2.0 ** -rng.integers(0, 3, size=n)
    sign = rng.choice([-1.0, 1.0], size=m)
    A = np.asfortranarray(np.stack([np.ones(m), -np.ones(m), sign * y, z], axis=1))
    B = np.asfortranarray(np.stack([np.ones(n), np.ones(n), x, w], axis=0))
    return A, B


@pytest.mark.parametrize("moduli", [16, 11, 8])
def test_crt_rounds_ties_and_sticky_bits_exactly(moduli):
    """C' on exact ties (rounded to even), one sticky bit above a tie, and every magnitude
    window of the rounding (with 16 moduli: |C'| from below 2^67 up to P/2; 11 and 8 moduli
    take the narrower windows): bit for bit the model, which rounds the exact integer once."""
    m, n, k = 96, 80, 4
    rng = np.random.default_rng(23)
    A, B = _rounding_operands(m, n, rng)
    model = crt_model()
    b = model.bits(moduli)
    _, Ai = model.scaled_integers(A, b)
    _, Bi = model.scaled_integers(B.T, b)
    Cp = Ai.dot(Bi.T)
    lengths = np.vectorize(lambda x: abs(int(x)).bit_length())(Cp)

    def tie(x):
        x = abs(int(x))
        L = x.bit_length()
        return L > 54 and x & ((1 << (L - 53)) - 1) == 1 << (L - 54)

    if moduli == 16:
        assert int(np.vectorize(tie)(Cp).sum()) >= 10
        assert (lengths >= 119).sum() > 0 and ((lengths >= 68) & (lengths < 119)).sum() > 0
        assert ((lengths > 0) & (lengths < 68)).sum() > 0
    eb.set_dgemm_moduli(moduli)
    eb.set_dgemm_tolerance(1.0)
    C = np.asfortranarray(rng.standard_normal((m, n)))
    for beta in (0.0, -0.5):
        rc, Cg = _device_call("N", "N", m, n, k, 1.0, A, m, B, k, beta, C, m, check=False)
        assert rc == eb.EB2_OK
        np.testing.assert_array_equal(Cg, _model(A, "N", B, "N", m, n, k, 1.0, beta, C, moduli))


@pytest.mark.parametrize("tile_n", [0, 1024])
def test_crt_long_k_accumulates_in_chunks(tile_n):
    """K beyond one exact INT32 unit (1023 x 128): the epilogue adds residues mod p (with the
    256 x 256 one-CTA tile, whose single accumulator is drained between the chunks)."""
    m, n, k = 3, 2, 1023 * 128 + 300
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, "T", "N", seed=9)
    eb.set_dgemm_tolerance(1.0)
    eb.set_tile_n(tile_n)
    Cg = C.copy(order="F")
    eb.dgemm("T", "N", m, n, k, 1.0, A, lda, B, ldb, 0.0, Cg, ldc)
    np.testing.assert_array_equal(Cg, _model(A, "T", B, "N", m, n, k, 1.0, 0.0, C, 16))


@pytest.mark.parametrize("r", [0, 8, 32])
def test_crt_accuracy_no_worse_than_native(r):
    m = n = k = 1024
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, "N", "N", pad=8, r=r, seed=200 + r)
    rng = np.random.default_rng(r)
    rows = np.sort(rng.choice(m, 48, replace=False))
    cols = np.sort(rng.choice(n, 48, replace=False))
    hi, lo = dd_reference("N", "N", m, n, k, 1.0, A, lda, B, ldb, 0.0, None, ldc, rows, cols)
    errs = {}
    for method in (eb.METHOD_NATIVE, eb.METHOD_CRT):
        eb.set_dgemm_method(method)
        Cg = C.copy(order="F")
        eb.dgemm("N", "N", m, n, k, 1.0, A, lda, B, ldb, 0.0, Cg, ldc)
        errs[method] = rel_error_vs_dd(Cg, hi, lo, rows, cols)
        if method == eb.METHOD_CRT:
            info = eb.last_call_info()
            assert info["method"] == eb.METHOD_CRT and 0.0 <= info["err_estimate"] <= U64
    assert errs[eb.METHOD_CRT] <= errs[eb.METHOD_NATIVE], errs
    assert errs[eb.METHOD_CRT] <= 2 * U64, errs


@pytest.mark.parametrize("beta", [0.0, -0.5])
def test_crt_escalation_adds_moduli(beta):
    """A target below what 16 moduli give: the check adds two moduli and the result is
    the 18-modulus model bit for bit (with beta != 0, C is written once, after the check)."""
    m, n, k = 96, 80, 1024
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, seed=17)
    eb.set_dgemm_tolerance(2.0 ** -60)
    Cg = C.copy(order="F")
    eb.dgemm("N", "N", m, n, k, 1.0, A, lda, B, ldb, beta, Cg, ldc)
    info = eb.last_call_info()
    assert info["escalations"] == 1 and info["slices"] == 18, info
    assert 0.0 < info["err_estimate"] <= 2.0 ** -60
    np.testing.assert_array_equal(Cg, _model(A, "N", B, "N", m, n, k, 1.0, beta, C, 18))
    # an unreachable target: 20 moduli, the result is still the 20-modulus product
    eb.set_dgemm_tolerance(2.0 ** -200)
    eb.clear_error()
    Cg = C.copy(order="F")
    eb.dgemm("N", "N", m, n, k, 1.0, A, lda, B, ldb, beta, Cg, ldc)
    info = eb.last_call_info()
    assert info["slices"] == 20 and eb.last_error()[0] == eb.EB2_ERR_ACCURACY
    np.testing.assert_array_equal(Cg, _model(A, "N", B, "N", m, n, k, 1.0, beta, C, 20))


def test_crt_host_and_device_entries_agree():
    m, n, k = 300, 200, 500
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, "T", "T", pad=2, seed=21)
    Ch = C.copy(order="F")
    eb.dgemm("T", "T", m, n, k, 0.5, A, lda, B, ldb, 2.0, Ch, ldc)
    rc, Cd = _device_call("T", "T", m, n, k, 0.5, A, lda, B, ldb, 2.0, C, ldc, check=True)
    assert rc == eb.EB2_OK
    np.testing.assert_array_equal(Ch, Cd)
    rc, Cn = _device_call("T", "T", m, n, k, 0.5, A, lda, B, ldb, 2.0, C, ldc, check=False)
    np.testing.assert_array_equal(Ch, Cn)


def test_crt_nonfinite_inputs_use_native_kernel():
    m, n, k = 50, 40, 30
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, seed=3)
    A[4, 7] = np.nan
    B[2, 9] = np.inf
    Cg = C.copy(order="F")
    eb.dgemm("N", "N", m, n, k, 1.0, A, lda, B, ldb, 0.0, Cg, ldc)
    assert eb.last_call_info()["nonfinite"] == 1
    eb.set_dgemm_method(eb.METHOD_NATIVE)
    Cn = C.copy(order="F")
    eb.dgemm("N", "N", m, n, k, 1.0, A, lda, B, ldb, 0.0, Cn, ldc)
    np.testing.assert_array_equal(np.isnan(Cg), np.isnan(Cn))
    fin = np.isfinite(Cn)
    np.testing.assert_array_equal(Cg[fin], Cn[fin])


def test_crt_beta_zero_ignores_nan_in_c():
    m, n, k = 64, 64, 64
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, seed=4)
    C[:] = np.nan
    eb.dgemm("N", "N", m, n, k, 1.0, A, lda, B, ldb, 0.0, C, ldc)
    assert np.all(np.isfinite(C[:m, :n]))
