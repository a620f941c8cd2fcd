"""Eigen's own Matrix operator*, compiled with EIGEN_USE_BLAS, runs on libeigen_b200.so.

tests/eigen_seam/eigen_seam_demo.cpp is built against the reference's Eigen headers
(tests/eigen_seam/Makefile) and linked with libeigen_b200.so first; this test runs it and
checks its self-verification plus the library's own call record."""
from __future__ import annotations

import json
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
DEMO = Path(__file__).resolve().parent / "eigen_seam" / "_bin" / "eigen_seam_demo"


@pytest.mark.parametrize("m,n,k", [(300, 200, 250), (1000, 517, 129)])
def test_eigen_operator_product_routes_to_library(m, n, k):
    if not DEMO.exists():
        pytest.fail(f"{DEMO} missing: build it with `make -C tests/eigen_seam if-present`")
    r = subprocess.run([str(DEMO), str(m), str(n), str(k)], capture_output=True, text=True, timeout=300)
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert line, r.stdout + r.stderr
    out = json.loads(line[-1])
    assert r.returncode == 0, out
    assert out["err_AB"] < 1e-14 and out["err_alpha_AtB"] < 1e-14 and out["err_float"] < 1e-5
    assert out["dgemm_launches"] > 0 and out["sgemm_launches"] > 0  # the products ran in the library
    # the default method: native for small products, otherwise the CRT emulation (>= 16 moduli)
    assert (out["dgemm_method"] == 1) or (out["dgemm_method"] == 3 and out["dgemm_slices"] >= 16)


SOLVERS = Path(__file__).resolve().parent / "eigen_seam" / "_bin" / "eigen_seam_solvers"


@pytest.mark.parametrize("n,rhs", [(600, 96), (1500, 300)])
def test_eigen_decompositions_route_level3_routines_to_library(n, rhs):
    """Eigen's blocked LLT and PartialPivLU, a triangular solve, a triangular product, a
    self-adjoint product, a rank update, a complex product, and complex LLT, triangular solve,
    triangular product and self-adjoint product, compiled with EIGEN_USE_BLAS: each result
    checks out and dtrsm_, dtrmm_, dsymm_, dsyrk_, dgemm_, zgemm_, ztrsm_, ztrmm_ and zhemm_ ran
    in the library (its per-routine counters)."""
    if not SOLVERS.exists():
        pytest.fail(f"{SOLVERS} missing: build it with `make -C tests/eigen_seam if-present`")
    r = subprocess.run([str(SOLVERS), str(n), str(rhs)], capture_output=True, text=True, timeout=600)
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert line, r.stdout + r.stderr
    out = json.loads(line[-1])
    assert r.returncode == 0, out
    for key in ("err_llt", "err_llt_solve", "err_trsm", "err_trmm", "err_symm", "err_syrk", "err_zgemm",
                "err_zllt_solve", "err_ztrsm", "err_ztrmm", "err_zhemm"):
        assert out[key] < 1e-13, (key, out)
    assert out["err_lu_solve"] < 1e-11, out
    assert all(v > 0 for v in out["calls"].values()), out
