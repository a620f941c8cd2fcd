"""Eigen's Tensor contractions on the GPU device run on libeigen_b200.so.

tests/eigen_tensor_gpu/tensor_contraction_gpu.cu is compiled with nvcc against a copy of the
reference's Eigen tree with include/eigen_b200/eigen_tensor_gpu_contraction.patch applied
(TensorContractionGpu.h gains a GEMM customisation point) and
include/eigen_b200/eigen_tensor_gpu_contraction.h, which specialises it for double and float
(tests/eigen_tensor_gpu/Makefile).  This test runs it: rank-2 contractions in all four
operand orientations, rank 3 over two index pairs, RowMajor, float, and a contraction that is
not a plain matrix product, each equal to Eigen's own CPU contraction (1e-13 relative for
double, 1e-5 for float), with exactly the plain products counted as library calls."""
from __future__ import annotations

import json
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
BIN = Path(__file__).resolve().parent / "eigen_tensor_gpu" / "_bin"


def _run(name, *args):
    demo = BIN / name
    if not demo.exists():
        pytest.fail(f"{demo} missing: build it with `make -C tests/eigen_tensor_gpu if-present`")
    r = subprocess.run([str(demo), *args], capture_output=True, text=True, timeout=600)
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert line, r.stdout + r.stderr
    return r.returncode, json.loads(line[-1])


def test_gpu_device_contractions_route_to_library():
    rc, out = _run("tensor_contraction_gpu")
    assert rc == 0, out
    assert out["worst_rel_err_double"] < 1e-13 and out["worst_rel_err_float"] < 1e-5, out
    assert out["library_calls"] == out["expected_calls"] == 7 and out["last_error"] == 0, out


def test_stock_gpu_contraction_still_correct_with_the_patch():
    """The patched tree without the library's specialisation: every contraction on Eigen's
    own kernels, same results."""
    rc, out = _run("tensor_contraction_gpu_stock")
    assert out["library_calls"] == 0, out
    assert out["worst_rel_err_double"] < 1e-13 and out["worst_rel_err_float"] < 1e-5, out
