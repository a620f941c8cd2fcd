"""eb2_dgemm_device_noalloc, the DGEMM entry point that allocates no device memory.

It exists for callers that cannot let a library call cudaMalloc -- a process whose GPU
memory belongs to another allocator (here: PyTorch's caching allocator holds the test's
buffers), or a path that must not allocate or free.  Its scratch is one fixed array in
device memory, shared by every call, so the test makes two different calls in a row and
checks both against the allocating entry point eb2_dgemm_device (same CRT method, 16
moduli, no accuracy check): the results must agree bit for bit, which is inside any
tolerance the other tests use.  It also checks the size limit and that the device's
free memory does not move across calls.

This file sorts last so that a run stopping at the first failure has run everything else.
"""
from __future__ import annotations

import numpy as np
import pytest

import eigen_b200 as eb
from _helpers import U64, gemm_error_bound, make_operands, op

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dev(x):
    """Column-major numpy matrix -> device tensor holding the same column-major bytes."""
    return torch.from_numpy(np.asfortranarray(x).T.copy()).cuda()


def _host(t):
    return np.asfortranarray(t.cpu().numpy().T)


@pytest.fixture(autouse=True)
def _gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    eb.load()
    eb.clear_error()
    yield
    eb.set_dgemm_method(eb.METHOD_AUTO)
    eb.set_dgemm_moduli(0)


CASES = [("N", "N", 700, 600, 500, 1.5, 0.5, 1), ("T", "N", 300, 900, 1000, -1.0, 0.0, 2)]


def _reference(ta, tb, m, n, k, alpha, beta, A, lda, B, ldb, C, ldc):
    """The allocating entry point on the same inputs, forced to the same method."""
    eb.set_dgemm_method(eb.METHOD_CRT)
    eb.set_dgemm_moduli(16)
    dC = _dev(C)
    rc = eb.dgemm_device(ta, tb, m, n, k, alpha, _dev(A), lda, _dev(B), ldb, beta, dC, ldc, check_accuracy=False)
    torch.cuda.synchronize()
    assert rc == eb.EB2_OK, eb.last_error()
    return _host(dC)


def test_noalloc_matches_allocating_entry_on_consecutive_calls():
    inputs = [make_operands(m, n, k, ta, tb, pad=2, seed=s) for (ta, tb, m, n, k, _, _, s) in CASES]
    refs = [_reference(ta, tb, m, n, k, al, be, *inp)
            for (ta, tb, m, n, k, al, be, _), inp in zip(CASES, inputs)]
    dev = [[_dev(x) for x in (A, B, C)] for (A, _, B, _, C, _) in inputs]
    torch.cuda.synchronize()
    for rep in range(2):  # every call reuses the scratch the previous call left behind
        for (ta, tb, m, n, k, al, be, _), (A, lda, B, ldb, C, ldc), (dA, dB, dC), ref in zip(CASES, inputs, dev, refs):
            dC.copy_(_dev(C))
            rc = eb.dgemm_device_noalloc(ta, tb, m, n, k, al, dA, lda, dB, ldb, be, dC, ldc)
            assert rc == eb.EB2_OK, eb.last_error()
            got = _host(dC)
            np.testing.assert_array_equal(got, ref)
            # and within the product error bound of the other tests
            want = al * (op(A, ta, m, k) @ op(B, tb, k, n)) + (be * C[:m, :n] if be else 0.0)
            bound = gemm_error_bound(A, ta, B, tb, m, n, k, al, be, C, U64)
            assert np.all(np.abs(got[:m, :n] - want) <= bound)


def test_noalloc_rejects_products_beyond_its_scratch_and_allocates_nothing():
    m = n = k = 512
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, seed=7)
    dA, dB, dC = _dev(A), _dev(B), _dev(C)
    assert eb.dgemm_device_noalloc("N", "N", m, n, k, 1.0, dA, lda, dB, ldb, 0.0, dC, ldc) == eb.EB2_OK
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        assert eb.dgemm_device_noalloc("N", "N", m, n, k, 1.0, dA, lda, dB, ldb, 0.0, dC, ldc) == eb.EB2_OK
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    # 2048^3 needs about 200 MB of scratch: refused before any launch, C untouched
    big = 2048
    x = torch.zeros((big, big), dtype=torch.float64, device="cuda")
    y = torch.full((big, big), 3.0, dtype=torch.float64, device="cuda")
    rc = eb.dgemm_device_noalloc("N", "N", big, big, big, 1.0, x, big, x, big, 0.0, y, big)
    assert rc == eb.EB2_ERR_ARG
    code, msg = eb.last_error()
    assert code == eb.EB2_ERR_ARG and "scratch" in msg
    assert bool(torch.all(y == 3.0))
    # dimensions whose scratch size would wrap the layout arithmetic are refused before it
    # (nothing is read: the refusal comes before any launch, so the small buffers suffice)
    eb.clear_error()
    huge = 1 << 31
    rc = eb.dgemm_device_noalloc("N", "N", huge, 8, huge, 1.0, x, huge, x, huge, 0.0, y, huge)
    assert rc == eb.EB2_ERR_ARG
    assert "scratch" in eb.last_error()[1]
    assert bool(torch.all(y == 3.0))
    # BLAS argument rules
    eb.clear_error()
    assert eb.dgemm_device_noalloc("X", "N", m, n, k, 1.0, dA, lda, dB, ldb, 0.0, dC, ldc) == eb.EB2_ERR_ARG
    assert eb.dgemm_device_noalloc("N", "N", m, n, k, 1.0, dA, m - 1, dB, ldb, 0.0, dC, ldc) == eb.EB2_ERR_ARG
