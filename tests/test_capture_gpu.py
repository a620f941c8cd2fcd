"""Stream-ordered products captured into a CUDA graph (GPU).

eb2_sgemm_device and eb2_dgemm_device without the accuracy check contain no host round trip,
so once a first call has sized the device workspace they can be captured on a stream and
replayed: every replay gives the bits of a direct call.  A DGEMM with the check needs the host
between kernels and refuses capture with EB2_ERR_ARG, leaving the capture usable.
"""
from __future__ import annotations

import pytest

import eigen_b200 as eb

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(autouse=True)
def _defaults():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    eb.load()
    eb.set_dgemm_method(eb.METHOD_AUTO)
    eb.set_sgemm_method(eb.METHOD_AUTO)
    eb.clear_error()
    yield
    eb.set_dgemm_method(eb.METHOD_AUTO)
    eb.set_sgemm_method(eb.METHOD_AUTO)
    eb.set_dgemm_moduli(0)


@pytest.mark.parametrize("dtype,method", [("s", eb.METHOD_AUTO), ("s", eb.METHOD_NATIVE), ("d", eb.METHOD_CRT),
                                          ("d", eb.METHOD_NATIVE)])
def test_capture_and_replay(dtype, method):
    (eb.set_dgemm_method if dtype == "d" else eb.set_sgemm_method)(method)
    # a captured call has no picker stage 2 (it needs the host): fix the modulus count so the
    # direct call makes the same choice
    eb.set_dgemm_moduli(16)
    tdt = torch.float64 if dtype == "d" else torch.float32
    m, n, k = 700, 520, 900
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    A = torch.rand((k, m), dtype=tdt, device="cuda", generator=g) * 2 - 1  # column-major m x k
    B = torch.rand((n, k), dtype=tdt, device="cuda", generator=g) * 2 - 1  # column-major k x n
    C0 = torch.rand((n, m), dtype=tdt, device="cuda", generator=g)
    s = torch.cuda.Stream()

    def call(C):
        if dtype == "d":
            return eb.dgemm_device("N", "N", m, n, k, 0.75, A, m, B, k, 0.5, C, m, stream=s.cuda_stream,
                                   check_accuracy=False)
        return eb.sgemm_device("N", "N", m, n, k, 0.75, A, m, B, k, 0.5, C, m, stream=s.cuda_stream)

    ref = C0.clone()
    with torch.cuda.stream(s):
        assert call(ref) == eb.EB2_OK
    s.synchronize()
    C = C0.clone()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        assert call(C) == eb.EB2_OK
    for _ in range(3):
        C.copy_(C0)
        graph.replay()
        torch.cuda.synchronize()
        assert torch.equal(C, ref)


def test_checked_dgemm_refuses_capture():
    S = 256
    A = torch.rand((S, S), dtype=torch.float64, device="cuda")
    C = torch.zeros((S, S), dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        assert eb.dgemm_device("N", "N", S, S, S, 1.0, A, S, A, S, 0.0, C, S, stream=s.cuda_stream,
                               check_accuracy=False) == eb.EB2_OK
    s.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        rc = eb.dgemm_device("N", "N", S, S, S, 1.0, A, S, A, S, 0.0, C, S, stream=s.cuda_stream,
                             check_accuracy=True)
        C.add_(1.0)  # the capture itself stays valid
    assert rc == eb.EB2_ERR_ARG
    assert "check_accuracy" in eb.last_error()[1]
    eb.clear_error()
    graph.replay()
    torch.cuda.synchronize()
