"""The C-ABI library loads and exports every symbol its header declares, and the
paths that need no GPU behave like Eigen's BLAS shim (CPU-only)."""
from __future__ import annotations

import ctypes
import re
import subprocess

import numpy as np
import pytest

import eigen_b200 as eb
from _helpers import golden, load_xerbla_recorder


def declared_functions() -> list[str]:
    text = eb.HEADER_PATH.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*([A-Za-z_][A-Za-z0-9_]*)\s*\(", text, re.M)
    return sorted(set(n for n in names if n not in ("if", "while", "return")))


def test_header_declares_blas_and_extensions():
    names = declared_functions()
    for n in ("dgemm_", "sgemm_", "dgemm_64_", "sgemm_64_", "xerbla_", "eb2_last_error", "eb2_dgemm_device"):
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = eb.load()
    out = subprocess.run(["nm", "-D", "--defined-only", str(eb.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    for name in declared_functions():
        assert name in exported, name
        assert hasattr(lib, name)


def test_xerbla_is_weak_in_the_library():
    out = subprocess.run(["nm", "-D", str(eb.LIB_PATH)], capture_output=True, text=True, check=True).stdout
    kinds = {line.split()[-1]: line.split()[-2] for line in out.splitlines() if len(line.split()) >= 2}
    assert kinds.get("xerbla_") == "W"


def test_library_is_sm100a_only_and_links_no_torch():
    out = subprocess.run(["ldd", str(eb.LIB_PATH)], capture_output=True, text=True).stdout
    assert "torch" not in out and "libcudart" not in out  # static CUDA runtime, no torch dependency


@pytest.mark.parametrize("ilp64", [False, True])
def test_argument_errors_match_reference_info_codes(ilp64):
    """Every argument-error case of the golden set gives the reference's info code
    through xerbla_ (blas/level3_impl.h:61-78) and touches nothing: no GPU needed."""
    rec = load_xerbla_recorder()
    _, errors = golden()
    dummy = np.zeros(64)
    for e in errors:
        rec.record_xerbla_reset()
        eb.dgemm(e["ta"], e["tb"], e["m"], e["n"], e["k"], 1.0, dummy, e["lda"], dummy, e["ldb"], 0.0, dummy,
                 e["ldc"], ilp64=ilp64)
        got = rec.record_xerbla_last_info() if rec.record_xerbla_calls() else 0
        assert got == e["info"], e
        if got:
            assert rec.record_xerbla_last_name().decode() == "DGEMM "
    rec.record_xerbla_reset()
    eb.sgemm("N", "N", 3, 2, 2, 1.0, dummy, 2, dummy, 2, 0.0, dummy, 3, ilp64=ilp64)
    assert rec.record_xerbla_last_info() == 8 and rec.record_xerbla_last_name().decode() == "SGEMM "


def test_quick_return_leaves_c_untouched():
    c = np.full(8, 7.0)
    a = np.full(8, np.nan)
    eb.dgemm("N", "N", 0, 2, 2, 1.0, a, 1, a, 2, 0.0, c, 1)
    eb.dgemm("N", "N", 2, 0, 2, 1.0, a, 2, a, 2, 0.0, c, 2)
    assert np.all(c == 7.0)


def test_setters_validate():
    assert eb.set_dgemm_slices(1) == eb.EB2_ERR_ARG
    assert eb.set_dgemm_slices(13) == eb.EB2_ERR_ARG
    assert eb.set_dgemm_slices(9) == eb.EB2_OK
    assert eb.set_dgemm_slices(0) == eb.EB2_OK
    assert eb.set_tile_n(64) == eb.EB2_ERR_ARG
    assert eb.set_tile_n(128) == eb.EB2_OK and eb.set_tile_n(0) == eb.EB2_OK
    assert eb.set_dgemm_tolerance(0.0) == eb.EB2_ERR_ARG
    assert eb.set_dgemm_tolerance(2.0 ** -53) == eb.EB2_OK
    assert eb.set_dgemm_method(7) == eb.EB2_ERR_ARG
    assert eb.set_dgemm_method(eb.METHOD_AUTO) == eb.EB2_OK
    assert "sm_100a" in eb.version()


def _has_cuda() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_cuda(), reason="checks the no-device path")
def test_no_device_is_reported_and_c_untouched():
    eb.clear_error()
    a = np.ones(4)
    c = np.full(4, 3.0)
    eb.dgemm("N", "N", 2, 2, 2, 1.0, a, 2, a, 2, 0.0, c, 2)
    code, msg = eb.last_error()
    assert code == eb.EB2_ERR_NO_DEVICE and msg
    assert np.all(c == 3.0)
    assert eb.dgemm_device("N", "N", 2, 2, 2, 1.0, 1, 2, 1, 2, 0.0, 1, 2) == eb.EB2_ERR_NO_DEVICE
    assert eb.dgemm_device("X", "N", 2, 2, 2, 1.0, 1, 2, 1, 2, 0.0, 1, 2) == eb.EB2_ERR_ARG
