"""The other level-3 routines' C ABI without a GPU: exported symbols, and the argument errors of
?gemmtr_, ?syrk_, ?syr2k_, ?symm_, ?trmm_, ?trsm_ and zgemm_/cgemm_ against the reference's info
codes and xerbla_ names (blas/level3_impl.h:12-754), recorded from the reference in
tests/golden/level3_golden.npz and tests/golden/complex_golden.npz.  Argument errors and n == 0
quick returns touch neither the device nor the operands."""
from __future__ import annotations

import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

import eigen_b200 as eb
from _helpers import load_xerbla_recorder

GOLDEN = Path(__file__).resolve().parent / "golden" / "level3_golden.npz"
COMPLEX_GOLDEN = Path(__file__).resolve().parent / "golden" / "complex_golden.npz"
ROUTINES = ("gemmtr", "syrk", "syr2k", "symm", "trmm", "trsm")


def _errors():
    z = np.load(GOLDEN)
    return json.loads(bytes(z["meta"]).decode())["errors"]


def test_every_level3_symbol_is_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", str(eb.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    for r in ROUTINES:
        for d in "ds":
            for sfx in ("_", "_64_"):
                assert d + r + sfx in exported
    for sfx in ("_", "_64_"):
        assert "zgemm" + sfx in exported and "cgemm" + sfx in exported


def test_golden_covers_every_info_code():
    codes = {}
    for e in _errors():
        codes.setdefault(e["routine"], set()).add(e["info"])
    assert codes["gemmtr"] == {0, 1, 2, 3, 4, 5, 8, 10, 13}
    assert codes["syrk"] == {0, 1, 2, 3, 4, 7, 10}
    assert codes["syr2k"] == {1, 2, 3, 4, 7, 9, 12}
    assert codes["symm"] == {0, 1, 2, 3, 4, 7, 9, 12}
    assert codes["trmm"] == codes["trsm"] == {0, 1, 2, 3, 4, 5, 6, 9, 11}


@pytest.mark.parametrize("ilp64", [False, True])
@pytest.mark.parametrize("dtype", ["d", "s"])
def test_argument_errors_match_reference(ilp64, dtype):
    rec = load_xerbla_recorder()
    npdt = np.float64 if dtype == "d" else np.float32
    sentinel = np.full(256, 7.0, dtype=npdt)
    for e in _errors():
        values = [sentinel if v is None else v for v in e["values"]]
        rec.record_xerbla_reset()
        eb.level3(dtype + e["routine"], *values, ilp64=ilp64)
        got = rec.record_xerbla_last_info() if rec.record_xerbla_calls() else 0
        assert got == e["info"], e
        if got:
            want = (dtype.upper() + e["name"][1:])
            assert rec.record_xerbla_last_name().decode() == want, e
        assert np.all(sentinel == 7.0)  # nothing written


def test_xerbla_lengths_follow_the_reference():
    """GEMMTR passes 7 characters (blas/level3_impl.h:199), the others 6."""
    rec = load_xerbla_recorder()
    a = np.zeros(16)
    rec.record_xerbla_reset()
    eb.level3("dgemmtr", "X", "N", "N", 2, 2, 1.0, a, 2, a, 2, 0.0, a, 2)
    assert rec.record_xerbla_last_name().decode() == "DGEMMTR"
    rec.record_xerbla_reset()
    eb.level3("strsm", "L", "U", "N", "N", 2, 2, 1.0, a, 1, a, 2)
    assert rec.record_xerbla_last_info() == 9 and rec.record_xerbla_last_name().decode() == "STRSM "



@pytest.mark.parametrize("ilp64", [False, True])
@pytest.mark.parametrize("dtype", ["z", "c"])
def test_complex_gemm_argument_errors_match_reference(ilp64, dtype):
    """zgemm_/cgemm_: the info codes of blas/level3_impl.h:61-78 recorded from the reference."""
    rec = load_xerbla_recorder()
    errors = json.loads(bytes(np.load(COMPLEX_GOLDEN)["meta"]).decode())["errors"]
    assert {e["info"] for e in errors} == {0, 1, 2, 3, 4, 5, 8, 10, 13}
    sentinel = np.full(64, 7 + 7j, dtype=np.complex128 if dtype == "z" else np.complex64)
    for e in errors:
        rec.record_xerbla_reset()
        eb.complex_gemm(dtype, e["ta"], e["tb"], e["m"], e["n"], e["k"], 1.0, sentinel, e["lda"], sentinel, e["ldb"],
                        0.0, sentinel, e["ldc"], ilp64=ilp64)
        got = rec.record_xerbla_last_info() if rec.record_xerbla_calls() else 0
        assert got == e["info"], e
        if got:
            assert rec.record_xerbla_last_name().decode() == dtype.upper() + "GEMM "
        assert np.all(sentinel == 7 + 7j)


CLEVEL3_GOLDEN = Path(__file__).resolve().parent / "golden" / "complex_level3_golden.npz"


@pytest.mark.parametrize("ilp64", [False, True])
@pytest.mark.parametrize("dtype", ["z", "c"])
def test_complex_level3_argument_errors_match_reference(ilp64, dtype):
    """z/c trsm_, trmm_, symm_, hemm_: the reference's info codes and xerbla_ names."""
    rec = load_xerbla_recorder()
    errors = json.loads(bytes(np.load(CLEVEL3_GOLDEN)["meta"]).decode())["errors"]
    sentinel = np.full(256, 7 + 7j, dtype=np.complex128 if dtype == "z" else np.complex64)
    seen = {}
    for e in errors:
        values = [sentinel if v is None else v for v in e["values"]]
        rec.record_xerbla_reset()
        eb.level3(dtype + e["routine"], *values, ilp64=ilp64)
        got = rec.record_xerbla_last_info() if rec.record_xerbla_calls() else 0
        assert got == e["info"], e
        if got:
            assert rec.record_xerbla_last_name().decode() == dtype.upper() + e["name"][1:], e
        seen.setdefault(e["routine"], set()).add(got)
        assert np.all(sentinel == 7 + 7j)
    assert seen["trsm"] == seen["trmm"] == {0, 1, 2, 3, 4, 5, 6, 9, 11}
    assert seen["hemm"] == seen["symm"] == {0, 1, 2, 3, 4, 7, 9, 12}
