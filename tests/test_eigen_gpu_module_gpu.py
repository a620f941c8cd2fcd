"""Eigen's gpu::DeviceMatrix GEMM expressions run on libeigen_b200.so.

tests/eigen_gpu/device_matrix_gemm.cpp is built against the reference's
unsupported/Eigen/GPU with include/eigen_b200/eigen_gpu_gemm.h, which specialises the
module's GEMM entry (Eigen::gpu::internal::cublaslt_gemm, CuBlasSupport.h:287-323) for
double and float (tests/eigen_gpu/Makefile).  This test runs it: every expression form of
DeviceDispatch.h:38-93 agrees with Eigen's CPU product, and the library's call record shows
the products ran in it."""
from __future__ import annotations

import json
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
DEMO = Path(__file__).resolve().parent / "eigen_gpu" / "_bin" / "device_matrix_gemm"


@pytest.mark.parametrize("m,n,k", [(700, 500, 600), (2048, 1024, 3000), (33, 17, 5)])
def test_device_matrix_gemm_routes_to_library(m, n, k):
    if not DEMO.exists():
        pytest.fail(f"{DEMO} missing: build it with `make -C tests/eigen_gpu if-present`")
    r = subprocess.run([str(DEMO), str(m), str(n), str(k)], capture_output=True, text=True, timeout=600)
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert line, r.stdout + r.stderr
    out = json.loads(line[-1])
    assert r.returncode == 0, out
    assert out["err_double"] < 1e-14 and out["err_float"] < 1e-5, out
    assert out["double_dtype"] == "d" and out["float_dtype"] == "s", out
    assert out["double_launches"] > 0 and out["float_launches"] > 0, out
