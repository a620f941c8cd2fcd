"""The BLAS entry's pipelined DGEMM on host buffers (copies overlapped with the CRT product
by column blocks) through the C ABI (GPU).

Every entry of the CRT product depends only on its row of op(A) and its column of op(B), so
the pipelined call must equal the device entry point bit for bit whatever the blocking:
transposes, beta != 0, padded leading dimensions, a ragged last block, per-block escalation
of the modulus count, NaN/Inf inputs.
"""
from __future__ import annotations

import numpy as np
import pytest

import eigen_b200 as eb
from _helpers import U64, make_operands

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(autouse=True)
def _defaults():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    eb.load()
    eb.set_dgemm_method(eb.METHOD_CRT)
    eb.set_dgemm_moduli(0)
    eb.set_dgemm_tolerance(U64)
    eb.set_tile_n(0)
    eb.clear_error()
    yield
    eb.set_dgemm_method(eb.METHOD_AUTO)
    eb.set_dgemm_moduli(0)
    eb.set_dgemm_tolerance(U64)


def _device(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, moduli=16, check=False):
    eb.set_dgemm_moduli(moduli)
    dev = [torch.from_numpy(np.asfortranarray(x).T.copy()).cuda() for x in (A, B, C)]
    rc = eb.dgemm_device(ta, tb, m, n, k, alpha, dev[0], lda, dev[1], ldb, beta, dev[2], ldc, check_accuracy=check)
    torch.cuda.synchronize()
    eb.set_dgemm_moduli(0)
    assert rc == eb.EB2_OK, eb.last_error()
    return np.asfortranarray(dev[2].cpu().numpy().T)


@pytest.mark.parametrize("ta,tb,m,n,k,beta", [("N", "N", 700, 2500, 600, 0.0), ("T", "N", 512, 1024, 300, 1.0),
                                               ("N", "T", 300, 1500, 1000, -0.5), ("T", "T", 257, 3100, 259, 2.0)])
def test_pipelined_host_call_equals_device_path(ta, tb, m, n, k, beta):
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, ta, tb, pad=5, r=3, seed=m + n)
    Ch = C.copy(order="F")
    eb.dgemm(ta, tb, m, n, k, 1.25, A, lda, B, ldb, beta, Ch, ldc)
    info = eb.last_call_info()
    assert info["method"] == eb.METHOD_CRT and info["staged"] == 1 and eb.last_error()[0] == eb.EB2_OK
    assert info["escalations"] == 0 and 0.0 <= info["err_estimate"] <= U64
    Cd = _device(ta, tb, m, n, k, 1.25, A, lda, B, ldb, beta, C, ldc)
    np.testing.assert_array_equal(Ch, Cd)  # padding rows of C untouched as well


@pytest.mark.parametrize("beta", [0.0, 0.75])
def test_pipelined_blocks_escalate_like_the_device_path(beta):
    """A target 16 moduli miss: every block is redone by the ordinary path with 18 moduli,
    from the host's C (beta != 0), and equals the 18-modulus product."""
    m, n, k = 300, 1100, 1024
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, seed=31)
    eb.set_dgemm_tolerance(2.0 ** -60)
    Ch = C.copy(order="F")
    eb.dgemm("N", "N", m, n, k, 1.0, A, lda, B, ldb, beta, Ch, ldc)
    info = eb.last_call_info()
    assert info["slices"] == 18 and info["escalations"] >= 1, info
    eb.set_dgemm_tolerance(1.0)
    np.testing.assert_array_equal(Ch, _device("N", "N", m, n, k, 1.0, A, lda, B, ldb, beta, C, ldc, moduli=18))


def test_pipelined_nonfinite_block_uses_native_kernel():
    m, n, k = 400, 2100, 300
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, seed=41)
    B[5, 1900] = np.inf  # a column in the last block
    Ch = C.copy(order="F")
    eb.dgemm("N", "N", m, n, k, 1.0, A, lda, B, ldb, 0.0, Ch, ldc)
    assert eb.last_call_info()["nonfinite"] == 1
    eb.set_dgemm_method(eb.METHOD_NATIVE)
    Cn = C.copy(order="F")
    eb.dgemm("N", "N", m, n, k, 1.0, A, lda, B, ldb, 0.0, Cn, ldc)
    np.testing.assert_array_equal(np.isinf(Ch), np.isinf(Cn))
    fin = np.isfinite(Cn)
    # blocks computed before the Inf was seen are CRT results; the rest are native
    assert np.max(np.abs(Ch[fin] - Cn[fin])) <= 1e-12 * np.max(np.abs(Cn[fin]))


@pytest.mark.parametrize("kinds", ["pageable", "pinned", "mixed"])
def test_pipelined_host_call_bounce_buffers(kinds):
    """Pageable host operands go through the library's pinned bounce buffers (16 MB chunks of
    whole columns, several per operand and per C block here, both directions), pinned ones
    straight to the copy engine: every mix gives the device path's bits."""
    m, n, k = 4096, 3000, 700
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, "N", "N", pad=3, r=2, seed=77)

    def host(x, pin):
        if not pin:
            return np.asfortranarray(x.copy())
        t = torch.empty(x.shape[::-1], dtype=torch.float64, pin_memory=True)  # column-major view
        t.copy_(torch.from_numpy(np.ascontiguousarray(x.T)))
        return t

    pins = {"pageable": (False, False, False), "pinned": (True, True, True), "mixed": (True, False, False)}[kinds]
    hA, hB, hC = host(A, pins[0]), host(B, pins[1]), host(C, pins[2])
    eb.dgemm("N", "N", m, n, k, 0.5, hA, lda, hB, ldb, 1.0, hC, ldc)
    assert eb.last_error()[0] == eb.EB2_OK, eb.last_error()
    assert eb.last_call_info()["staged"] == 1
    got = np.asfortranarray(hC.numpy().T) if isinstance(hC, torch.Tensor) else hC
    np.testing.assert_array_equal(got, _device("N", "N", m, n, k, 0.5, A, lda, B, ldb, 1.0, C, ldc))
