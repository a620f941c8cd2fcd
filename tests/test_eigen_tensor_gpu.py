"""Eigen's Tensor contractions (double) run on libeigen_b200.so.

tests/eigen_tensor/tensor_contraction.cpp is built against the reference's
unsupported/Eigen/Tensor with include/eigen_b200/eigen_tensor_contraction.h, which
specialises the contraction's blocking and kernel (TensorContraction.h:128-157) so that each
double contraction is one dgemm_ call into the library (tests/eigen_tensor/Makefile).  This
test runs it: contractions of rank 2..4 over one and two index pairs, on the default device,
on a thread pool and inside a larger expression, all equal to a direct long-double loop
within 1e-14 relative, and the library's dgemm_ counter shows they ran in it."""
from __future__ import annotations

import json
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
DEMO = Path(__file__).resolve().parent / "eigen_tensor" / "_bin" / "tensor_contraction"


def test_tensor_contractions_route_to_library():
    if not DEMO.exists():
        pytest.fail(f"{DEMO} missing: build it with `make -C tests/eigen_tensor if-present`")
    r = subprocess.run([str(DEMO)], capture_output=True, text=True, timeout=600)
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert line, r.stdout + r.stderr
    out = json.loads(line[-1])
    assert r.returncode == 0, out
    assert out["worst_rel_err"] < 1e-14 and out["dgemm_calls"] >= 5 and out["last_error"] == 0, out
