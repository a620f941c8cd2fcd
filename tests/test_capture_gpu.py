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


@pytest.mark.parametrize("dtype", ["d", "s"])
def test_replay_after_workspace_growth(dtype):
    """A graph keeps the workspace address it captured: a later direct call that needs a larger
    workspace must not free it under the graph, so replays still give the direct call's bits."""
    eb.set_dgemm_method(eb.METHOD_CRT)
    eb.set_dgemm_moduli(16)
    tdt = torch.float64 if dtype == "d" else torch.float32
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    s = torch.cuda.Stream()

    def call(m, n, k, A, B, C):
        if dtype == "d":
            return eb.dgemm_device("N", "N", m, n, k, 1.25, A, m, B, k, 0.5, C, m, stream=s.cuda_stream,
                                   check_accuracy=False)
        return eb.sgemm_device("N", "N", m, n, k, 1.25, A, m, B, k, 0.5, C, m, stream=s.cuda_stream)

    m, n, k = 700, 520, 900
    A = torch.rand((k, m), dtype=tdt, device="cuda", generator=g) * 2 - 1
    B = torch.rand((n, k), dtype=tdt, device="cuda", generator=g) * 2 - 1
    C0 = torch.rand((n, m), dtype=tdt, device="cuda", generator=g)
    ref = C0.clone()
    with torch.cuda.stream(s):
        assert call(m, n, k, A, B, ref) == eb.EB2_OK
    s.synchronize()
    C = C0.clone()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        assert call(m, n, k, A, B, C) == eb.EB2_OK
    # a direct call large enough to grow the workspace past anything sized so far
    S = 6144
    A2 = torch.rand((S, S), dtype=tdt, device="cuda", generator=g) * 2 - 1
    C2 = torch.zeros((S, S), dtype=tdt, device="cuda")
    with torch.cuda.stream(s):
        assert call(S, S, S, A2, A2, C2) == eb.EB2_OK
    s.synchronize()
    del A2, C2
    for _ in range(2):
        C.copy_(C0)
        graph.replay()
        torch.cuda.synchronize()
        assert torch.equal(C, ref)
    # and the large product's workspace serves direct calls of the small size as well
    C3 = C0.clone()
    with torch.cuda.stream(s):
        assert call(m, n, k, A, B, C3) == eb.EB2_OK
    s.synchronize()
    assert torch.equal(C3, ref)


_FIRST_CAPTURE = r"""
import torch, eigen_b200 as eb
eb.load()
S = 1024
A = torch.rand((S, S), dtype=torch.float64, device="cuda")
C = torch.zeros((S, S), dtype=torch.float64, device="cuda")
s = torch.cuda.Stream()

def captured(expect):
    C.zero_()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        rc = eb.dgemm_device("N", "N", S, S, S, 1.0, A, S, A, S, 0.0, C, S, stream=s.cuda_stream,
                             check_accuracy=False)
        C.add_(1.0)  # the capture itself stays valid
    assert rc == eb.EB2_ERR_ARG, rc
    assert expect in eb.last_error()[1], eb.last_error()
    eb.clear_error()
    graph.replay()
    torch.cuda.synchronize()
    assert torch.all(C == 1.0)

# no context on the device yet: creating it would allocate inside the capture
captured("direct call first")
# a context, but no workspace yet (the native method needs none)
eb.set_dgemm_method(eb.METHOD_NATIVE)
with torch.cuda.stream(s):
    assert eb.dgemm_device("N", "N", 64, 64, 64, 1.0, A, S, A, S, 0.0, C, S, stream=s.cuda_stream,
                           check_accuracy=False) == eb.EB2_OK
s.synchronize()
eb.set_dgemm_method(eb.METHOD_CRT)
eb.set_dgemm_moduli(16)
captured("direct call of this size first")
with torch.cuda.stream(s):
    assert eb.dgemm_device("N", "N", S, S, S, 1.0, A, S, A, S, 0.0, C, S, stream=s.cuda_stream,
                           check_accuracy=False) == eb.EB2_OK
s.synchronize()
ref = C.clone()
g2 = torch.cuda.CUDAGraph()
with torch.cuda.graph(g2, stream=s):
    assert eb.dgemm_device("N", "N", S, S, S, 1.0, A, S, A, S, 0.0, C, S, stream=s.cuda_stream,
                           check_accuracy=False) == eb.EB2_OK
C.zero_()
g2.replay()
torch.cuda.synchronize()
assert torch.equal(C, ref)
print("ok")
"""


def test_capture_before_any_direct_call_refuses():
    """In a fresh process neither the device context nor the workspace exists: a captured call
    must not create them inside the capture (the allocations would invalidate it) and returns
    EB2_ERR_ARG instead, leaving the capture valid; after a direct call of the same size the
    capture works."""
    import subprocess
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    r = subprocess.run([sys.executable, "-c", _FIRST_CAPTURE], cwd=root, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
