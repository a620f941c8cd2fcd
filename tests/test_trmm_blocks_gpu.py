"""DTRMM as one CRT product that skips the triangle's zero K blocks (GPU).

From 1024 rows up, with the emulated DGEMM, dtrmm expands the triangle (zeros outside, unit
diagonal when asked) and runs one CRT product; each output tile walks only the 128-wide K
blocks the triangle can make nonzero for it.  Leaving out blocks of zero residues changes no
bit, so for every side, triangle, transpose and diagonal the result equals, bit for bit, a
plain CRT DGEMM of the expanded triangle, and stays within the product error bound of an FP64
reference.
"""
from __future__ import annotations

import itertools

import numpy as np
import pytest

import eigen_b200 as eb
from _helpers import U64, gemm_error_bound

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(autouse=True)
def _defaults():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    eb.load()
    eb.set_dgemm_method(eb.METHOD_CRT)
    eb.set_dgemm_tolerance(U64)
    eb.clear_error()
    yield
    eb.set_dgemm_method(eb.METHOD_AUTO)


@pytest.mark.parametrize("side,uplo,trans,diag", list(itertools.product("LR", "UL", "NTC", "NU")))
def test_trmm_equals_the_dense_product(side, uplo, trans, diag):
    rng = np.random.default_rng(hash((side, uplo, trans, diag)) % 2**32)
    size, other = 1100, 300
    m, n = (size, other) if side == "L" else (other, size)
    A = np.asfortranarray(rng.uniform(-1, 1, (size + 3, size)))
    B = np.asfortranarray(rng.uniform(-1, 1, (m + 2, n)))
    T = np.triu(A[:size, :size]) if uplo == "U" else np.tril(A[:size, :size])
    if diag == "U":
        np.fill_diagonal(T, 1.0)
    T = np.asfortranarray(T)
    alpha = 0.75
    got = B.copy(order="F")
    eb.level3("dtrmm", side, uplo, trans, diag, m, n, alpha, A, A.shape[0], got, got.shape[0])
    assert eb.last_error()[0] == eb.EB2_OK, eb.last_error()
    # the same product as a dense CRT DGEMM of the expanded triangle
    C = np.zeros((m, n), order="F")
    if side == "L":
        eb.dgemm(trans, "N", m, n, m, alpha, T, size, B, B.shape[0], 0.0, C, m)
    else:
        eb.dgemm("N", trans, m, n, n, alpha, B, B.shape[0], T, size, 0.0, C, m)
    assert eb.last_error()[0] == eb.EB2_OK, eb.last_error()
    np.testing.assert_array_equal(got[:m, :n], C)
    np.testing.assert_array_equal(got[m:, :], B[m:, :])
    opT = T.T if trans != "N" else T
    want = alpha * (opT @ B[:m, :n] if side == "L" else B[:m, :n] @ opT)
    if side == "L":
        bound = gemm_error_bound(opT, "N", B, "N", m, n, m, alpha, 0.0, None, U64)
    else:
        bound = gemm_error_bound(B, "N", opT, "N", m, n, n, alpha, 0.0, None, U64)
    assert np.all(np.abs(got[:m, :n] - want) <= 2 * bound)
