"""The bounded-wait error path of the tcgen05 GEMM, run on the device (GPU).

Every pipeline wait in the GEMM kernels is bounded in wall time.  With the bound set to
200 ns, the first waits of every CTA (a TMA copy landing, a unit's MMAs finishing) run out:
the kernel records the timeout in its status word, raises its abort flag, lets the copies and
MMAs already issued finish, frees its tensor memory and returns.  The call must report
EB2_ERR_TIMEOUT (no fault, no hang), and the next call with the default bound on the same
context must give the same bits as before.  One-CTA tiles only: there each CTA's producer
waits for its own copies before the CTA exits.
"""
from __future__ import annotations

import numpy as np
import pytest

import eigen_b200 as eb
from _helpers import make_operands

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(autouse=True)
def _defaults():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    eb.load()
    eb.clear_error()
    yield
    eb.set_wait_limit_ns(0)
    eb.set_tile_n(0)
    eb.set_dgemm_method(eb.METHOD_AUTO)
    eb.set_sgemm_method(eb.METHOD_AUTO)
    eb.set_dgemm_moduli(0)
    eb.set_dgemm_tolerance(2.0 ** -53)
    eb.clear_error()


def _run(dtype, A, lda, B, ldb, C, ldc, m, n, k):
    got = C.copy(order="F")
    (eb.dgemm if dtype == "d" else eb.sgemm)("N", "N", m, n, k, 1.0, A, lda, B, ldb, 0.5, got, ldc)
    return got, eb.last_error()


@pytest.mark.parametrize("dtype,tile", [("d", 256), ("d", 1024), ("s", 256), ("s", 128)])
def test_short_wait_limit_times_out_and_context_recovers(dtype, tile):
    if dtype == "d":
        eb.set_dgemm_method(eb.METHOD_CRT)
        eb.set_dgemm_moduli(16)
        eb.set_dgemm_tolerance(1.0)  # no escalation: one GEMM launch per call
    else:
        eb.set_sgemm_method(eb.METHOD_EMULATED)
    eb.set_tile_n(tile)
    m = n = k = 1024
    npdt = np.float64 if dtype == "d" else np.float32
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, pad=4, seed=91, dtype=npdt)
    ref, err = _run(dtype, A, lda, B, ldb, C, ldc, m, n, k)
    assert err[0] == eb.EB2_OK, err

    assert eb.set_wait_limit_ns(200) == eb.EB2_OK
    eb.clear_error()
    _, err = _run(dtype, A, lda, B, ldb, C, ldc, m, n, k)
    assert err[0] == eb.EB2_ERR_TIMEOUT, err
    assert "timed out" in err[1]
    torch.cuda.synchronize()  # the kernels returned: the device still answers

    eb.set_wait_limit_ns(0)
    eb.clear_error()
    for _ in range(2):
        again, err = _run(dtype, A, lda, B, ldb, C, ldc, m, n, k)
        assert err[0] == eb.EB2_OK, err
        np.testing.assert_array_equal(again, ref)


def test_wait_limit_rejects_negative():
    assert eb.set_wait_limit_ns(-1) == eb.EB2_ERR_ARG
