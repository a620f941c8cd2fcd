"""Concurrent callers of the library (GPU).

* host threads calling the BLAS entry (host buffers) and the device entry (device buffers,
  each thread on its own torch stream) at the same time: every result is within the GEMM
  error bound of its own reference, the sticky error and the call record stay per thread
  (an argument error planted in one thread is seen by that thread only);
* stream-ordered calls without the accuracy check, issued back to back on two streams with
  no synchronisation between them: they share the device's workspace, so the second must
  wait for the first on the GPU; both results equal those of the same calls made one at a
  time (bit for bit: the same kernels on the same data).
"""
from __future__ import annotations

import threading

import numpy as np
import pytest

import eigen_b200 as eb
from _helpers import U64, gemm_error_bound, make_operands, op

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(autouse=True)
def _defaults():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    eb.load()
    eb.set_dgemm_method(eb.METHOD_AUTO)
    eb.set_dgemm_tolerance(U64)
    eb.clear_error()
    yield
    eb.set_dgemm_method(eb.METHOD_AUTO)


def _check(A, ta, B, tb, m, n, k, alpha, beta, C0, got):
    want = alpha * (op(A, ta, m, k) @ op(B, tb, k, n)) + beta * C0[:m, :n]
    bound = gemm_error_bound(A, ta, B, tb, m, n, k, alpha, beta, C0, U64)
    # |got - exact| and |numpy - exact| are both within the bound
    assert np.all(np.abs(got[:m, :n] - want) <= 2 * bound)


def test_threads_share_the_device():
    shapes = [(300, 200, 257, "N", "T"), (129, 400, 64, "T", "N"), (512, 512, 512, "N", "N"),
              (77, 33, 1000, "T", "T"), (640, 96, 300, "N", "N"), (256, 256, 1024, "T", "N")]
    errors: list = []
    seen: dict = {}
    start = threading.Barrier(len(shapes) + 1)

    def worker(idx, m, n, k, ta, tb):
        try:
            A, lda, B, ldb, C, ldc = make_operands(m, n, k, ta, tb, pad=1, seed=100 + idx)
            device = idx % 2 == 1
            stream = torch.cuda.Stream() if device else None
            start.wait()
            for rep in range(3):
                alpha, beta = 1.25, (0.5 if rep != 1 else 0.0)
                if device:
                    dev = [torch.from_numpy(np.asfortranarray(x).T.copy()).cuda() for x in (A, B, C)]
                    torch.cuda.current_stream().synchronize()
                    rc = eb.dgemm_device(ta, tb, m, n, k, alpha, dev[0], lda, dev[1], ldb, beta, dev[2], ldc,
                                         stream=stream.cuda_stream, check_accuracy=rep != 2)
                    assert rc == eb.EB2_OK, (idx, rc, eb.last_error())
                    stream.synchronize()
                    got = np.asfortranarray(dev[2].cpu().numpy().T)
                else:
                    got = C.copy(order="F")
                    eb.dgemm(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, got, ldc)
                assert eb.last_error()[0] == eb.EB2_OK, (idx, eb.last_error())
                _check(A, ta, B, tb, m, n, k, alpha, beta, C, got)
            seen[idx] = eb.last_error()[0]
        except Exception as e:  # noqa: BLE001 - reported below
            errors.append((idx, repr(e)))

    def bad_caller():
        try:
            start.wait()
            for _ in range(5):
                rc = eb.dgemm_device("N", "N", -1, 4, 4, 1.0, None, 1, None, 1, 0.0, None, 1)
                assert rc == eb.EB2_ERR_ARG
            seen["bad"] = eb.last_error()[0]
        except Exception as e:  # noqa: BLE001
            errors.append(("bad", repr(e)))

    threads = [threading.Thread(target=worker, args=(i, *s)) for i, s in enumerate(shapes)]
    threads.append(threading.Thread(target=bad_caller))
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=600)
    assert not errors, errors
    assert seen.pop("bad") == eb.EB2_ERR_ARG
    assert len(seen) == len(shapes) and all(v == eb.EB2_OK for v in seen.values())
    assert eb.last_error()[0] == eb.EB2_OK  # this thread made no failing call


@pytest.mark.parametrize("method", [eb.METHOD_CRT, eb.METHOD_NATIVE])
def test_stream_ordered_calls_on_two_streams(method):
    eb.set_dgemm_method(method)
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    S = 2048
    mats = [torch.rand((S, S), dtype=torch.float64, device="cuda", generator=g) * 2 - 1 for _ in range(4)]
    # one at a time
    ref = []
    for i in range(2):
        C = torch.zeros((S, S), dtype=torch.float64, device="cuda")
        assert eb.dgemm_device("N", "N", S, S, S, 1.0, mats[2 * i], S, mats[2 * i + 1], S, 0.0, C, S,
                               check_accuracy=False) == eb.EB2_OK
        torch.cuda.synchronize()
        ref.append(C)
    # back to back on two streams, no synchronisation in between
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    outs = [torch.full((S, S), float("nan"), dtype=torch.float64, device="cuda") for _ in range(2)]
    torch.cuda.synchronize()
    for rep in range(3):
        for i, s in enumerate((s1, s2)):
            assert eb.dgemm_device("N", "N", S, S, S, 1.0, mats[2 * i], S, mats[2 * i + 1], S, 0.0, outs[i], S,
                                   stream=s.cuda_stream, check_accuracy=False) == eb.EB2_OK
    torch.cuda.synchronize()
    for i in range(2):
        assert torch.equal(outs[i], ref[i])
