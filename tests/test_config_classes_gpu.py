"""Configuration classes of the product path (GPU): each forced class runs the configuration it
names, and the classes of one method agree.

The CRT classes (one CTA or CTA pair, column-major or raster-group tile order, K split over
several work items) schedule the same exact integer products differently: modulo each p the
split residues add to the unsplit one, so every class gives the same bits.  The split-K class
really splits when the output tiles and moduli leave most SMs idle.  The SGEMM classes (FFMA,
split-BF16 on three tile shapes) and the grouped classes meet the usual error bounds.
"""
from __future__ import annotations

import numpy as np
import pytest

import eigen_b200 as eb
from _helpers import U32, U64, gemm_error_bound, make_operands

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(autouse=True)
def _defaults():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    eb.load()
    eb.clear_error()
    yield
    eb.set_config(-1)
    eb.set_dgemm_method(eb.METHOD_AUTO)
    eb.set_sgemm_method(eb.METHOD_AUTO)
    eb.set_dgemm_moduli(0)
    eb.set_dgemm_tolerance(2.0 ** -53)


def _dev(x):
    return torch.from_numpy(np.asfortranarray(x).T.copy()).cuda()


def _host(t):
    return np.asfortranarray(t.cpu().numpy().T)


@pytest.mark.parametrize("m,n,k,ta,tb,beta", [(200, 136, 20000, "N", "N", 0.0), (300, 260, 9000, "T", "N", 0.5),
                                               (700, 520, 900, "N", "T", 1.0), (130, 33, 4100, "T", "T", -1.5)])
def test_crt_classes_same_bits(m, n, k, ta, tb, beta):
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, ta, tb, pad=3, r=5, seed=m + n)
    dA, dB = _dev(A), _dev(B)
    eb.set_dgemm_moduli(16)
    results, infos = {}, {}
    for cfg in (1, 2, 3, 4, 5):
        assert eb.set_config(cfg) == eb.EB2_OK
        dC = _dev(C)
        rc = eb.dgemm_device(ta, tb, m, n, k, 1.25, dA, lda, dB, ldb, beta, dC, ldc, check_accuracy=True)
        torch.cuda.synchronize()
        assert rc == eb.EB2_OK, eb.last_error()
        results[cfg] = _host(dC)
        infos[cfg] = eb.last_call_info()
        assert infos[cfg]["config"] == cfg or (cfg == 5 and infos[cfg]["splits"] == 1), infos[cfg]
    for cfg in (2, 3, 4, 5):
        np.testing.assert_array_equal(results[cfg], results[1], err_msg=f"class {cfg}")
    # one-CTA classes: 256 x 256 tiles where padding the rows to 256 costs little, else 128 x 256
    cheap = ((m + 127) // 128) % 2 == 0 or m >= 2048
    assert infos[2]["tile_n"] == 512 and infos[1]["tile_n"] == (1024 if cheap else 256)
    # small outputs with long K: the split-K class splits
    if m * n <= 300 * 260:
        assert infos[5]["splits"] > 1, infos[5]
    want = 1.25 * (A[:m, :k] if ta == "N" else A[:k, :m].T) @ (B[:k, :n] if tb == "N" else B[:n, :k].T)
    want = want + (beta * C[:m, :n] if beta else 0.0)
    bound = gemm_error_bound(A, ta, B, tb, m, n, k, 1.25, beta, C, U64)
    assert np.all(np.abs(results[1][:m, :n] - want) <= bound)


def test_split_k_with_escalation_and_forced_native():
    """Split K through the a-posteriori check's added moduli (beta != 0 restarts from the old C),
    and class 0 forcing the native kernel."""
    m, n, k = 96, 80, 30000
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, pad=1, r=20, seed=5)
    dA, dB = _dev(A), _dev(B)
    eb.set_dgemm_moduli(8)
    eb.set_dgemm_tolerance(2.0 ** -53)
    eb.set_config(5)
    dC = _dev(C)
    assert eb.dgemm_device("N", "N", m, n, k, 1.0, dA, lda, dB, ldb, 0.75, dC, ldc, check_accuracy=True) == eb.EB2_OK
    torch.cuda.synchronize()
    info = eb.last_call_info()
    assert info["splits"] > 1 and info["escalations"] > 0, info
    split = _host(dC)
    eb.set_config(1)
    dC = _dev(C)
    assert eb.dgemm_device("N", "N", m, n, k, 1.0, dA, lda, dB, ldb, 0.75, dC, ldc, check_accuracy=True) == eb.EB2_OK
    torch.cuda.synchronize()
    assert eb.last_call_info()["slices"] == info["slices"]
    np.testing.assert_array_equal(split, _host(dC))
    eb.set_config(0)
    dC = _dev(C)
    assert eb.dgemm_device("N", "N", m, n, k, 1.0, dA, lda, dB, ldb, 0.75, dC, ldc, check_accuracy=True) == eb.EB2_OK
    torch.cuda.synchronize()
    assert eb.last_call_info()["method"] == eb.METHOD_NATIVE
    bound = gemm_error_bound(A, "N", B, "N", m, n, k, 1.0, 0.75, C, U64)
    assert np.all(np.abs(_host(dC)[:m, :n] - split[:m, :n]) <= 2 * bound)


@pytest.mark.parametrize("cfg", [6, 7, 8, 9])
def test_sgemm_classes(cfg):
    m, n, k = 333, 270, 1500
    A, lda, B, ldb, C, ldc = make_operands(m, n, k, "T", "N", pad=2, seed=cfg, dtype=np.float32)
    eb.set_config(cfg)
    dC = _dev(C)
    assert eb.sgemm_device("T", "N", m, n, k, 1.5, _dev(A), lda, _dev(B), ldb, 0.5, dC, ldc) == eb.EB2_OK
    torch.cuda.synchronize()
    info = eb.last_call_info()
    assert info["config"] == cfg, info
    assert info["method"] == (eb.METHOD_NATIVE if cfg == 6 else eb.METHOD_EMULATED)
    A64, B64, C64 = (x.astype(np.float64) for x in (A, B, C))
    want = 1.5 * A64[:k, :m].T @ B64[:k, :n] + 0.5 * C64[:m, :n]
    bound = gemm_error_bound(A64, "T", B64, "N", m, n, k, 1.5, 0.5, C64, U32)
    assert np.all(np.abs(_host(dC)[:m, :n] - want) <= bound)
