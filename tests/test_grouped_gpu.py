"""Grouped (batched) GEMM: one persistent, graph-captured launch for many uneven
products, checked against the oracle; FP64 bit for bit against one plain native DGEMM call
per product (same arithmetic, same order), FP32 (split-BF16 on the tensor cores) bit for bit
against the per-product launches of the same arithmetic and no less accurate than the FP32
FFMA kernel.  Small products share a warp (four of at most 8 x 8, two of at most 16 x 16);
the arithmetic of each output does not depend on that, so every class setting gives the
same bits."""
from __future__ import annotations

import numpy as np
import pytest

import eigen_b200 as eb
from _helpers import P, U32, U64, ch, gemm_error_bound, oracle, op_shape

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
    eb.set_grouped_classes(-1, -1)


def batch_sizes(count, seed, lo=3, hi=256):
    """Each of m, n, k = round(exp(U[ln lo, ln hi])); with probability 0.2 all three from {3,4,6,8}."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        if rng.random() < 0.2:
            s = int(rng.choice([3, 4, 6, 8]))
            out.append((s, s, s))
        else:
            out.append(tuple(int(round(np.exp(rng.uniform(np.log(lo), np.log(hi))))) for _ in range(3)))
    return out


def make_batch(sizes, dtype, seed, mixed=True):
    rng = np.random.default_rng(seed)
    npdt = np.float64 if dtype == "d" else np.float32
    host = []
    for i, (m, n, k) in enumerate(sizes):
        ta = "N" if not mixed else "NTC"[i % 3]
        tb = "N" if not mixed else "NT"[(i // 3) % 2]
        pad = 0 if not mixed else i % 4
        ar, ac = op_shape(ta, m, k)
        br, bc = op_shape(tb, k, n)
        A = np.asfortranarray(rng.uniform(-1, 1, (max(1, ar + pad), max(ac, 1))).astype(npdt))
        B = np.asfortranarray(rng.uniform(-1, 1, (max(1, br + pad), max(bc, 1))).astype(npdt))
        C = np.asfortranarray(rng.uniform(-1, 1, (max(1, m + pad), max(n, 1))).astype(npdt))
        alpha, beta = ((1.0, 0.0) if not mixed else [(1.0, 0.0), (1.5, 0.5), (0.0, 1.3), (-0.7, 1.0)][i % 4])
        host.append(dict(transa=ta, transb=tb, m=m, n=n, k=k, alpha=alpha, beta=beta, A=A, lda=max(1, ar + pad), B=B,
                         ldb=max(1, br + pad), C=C, ldc=max(1, m + pad)))
    return host


def to_device(host):
    dev, probs = [], []
    for h in host:
        tA = torch.from_numpy(h["A"].T.copy()).cuda()
        tB = torch.from_numpy(h["B"].T.copy()).cuda()
        tC = torch.from_numpy(h["C"].T.copy()).cuda()
        dev.append((tA, tB, tC))
        probs.append(dict(h, a=tA, b=tB, c=tC))
    return dev, probs


def back(t):
    return np.asfortranarray(t.cpu().numpy().T)


@pytest.mark.parametrize("dtype", ["d", "s"])
def test_grouped_matches_oracle_and_plain_calls(dtype):
    sizes = batch_sizes(300, seed=1)
    host = make_batch(sizes, dtype, seed=2)
    dev, probs = to_device(host)
    plan = eb.GroupedPlan(dtype, probs)
    assert plan.execute() == eb.EB2_OK
    torch.cuda.synchronize()
    lib = oracle()
    eps = U64 if dtype == "d" else U32
    f_native = eb.dgemm if dtype == "d" else eb.sgemm
    if dtype == "d":
        eb.set_dgemm_method(eb.METHOD_NATIVE)
    else:
        eb.set_sgemm_method(eb.METHOD_NATIVE)
    for h, (tA, tB, tC) in zip(host, dev):
        got = back(tC)
        ref = h["C"].copy(order="F")
        f = lib.oracle_dgemm if dtype == "d" else lib.oracle_sgemm
        f(ch(h["transa"]), ch(h["transb"]), h["m"], h["n"], h["k"], h["alpha"], P(h["A"]), h["lda"], P(h["B"]),
          h["ldb"], h["beta"], P(ref), h["ldc"])
        m, n = h["m"], h["n"]
        bound = gemm_error_bound(h["A"], h["transa"], h["B"], h["transb"], m, n, h["k"], h["alpha"], h["beta"],
                                 h["C"], eps)
        assert np.all(np.abs(got[:m, :n] - ref[:m, :n]) <= bound)
        np.testing.assert_array_equal(got[m:, :], h["C"][m:, :])
        if dtype == "d":  # one plain call of the native kernel gives the same bits
            plain = h["C"].copy(order="F")
            f_native(h["transa"], h["transb"], m, n, h["k"], h["alpha"], h["A"], h["lda"], h["B"], h["ldb"],
                     h["beta"], plain, h["ldc"])
            np.testing.assert_array_equal(got, plain)


def test_grouped_plan_replays_and_accumulates():
    sizes = batch_sizes(50, seed=3)
    host = make_batch(sizes, "d", seed=4, mixed=False)
    for h in host:
        h["beta"] = 1.0
        h["C"][:] = 0.0
    dev, probs = to_device(host)
    plan = eb.GroupedPlan("d", probs)
    s = torch.cuda.Stream()
    for _ in range(3):
        assert plan.execute(s.cuda_stream) == eb.EB2_OK
    s.synchronize()
    for h, (tA, tB, tC) in zip(host, dev):
        one = np.zeros_like(h["C"])
        oracle().oracle_dgemm(b"N", b"N", h["m"], h["n"], h["k"], 1.0, P(h["A"]), h["lda"], P(h["B"]), h["ldb"], 0.0,
                              P(one), h["ldc"])
        np.testing.assert_allclose(back(tC), 3 * one, rtol=1e-12, atol=1e-12)


def test_grouped_blas_edge_rules():
    host = make_batch([(5, 4, 3), (6, 6, 0), (0, 5, 5), (7, 3, 2)], "d", seed=5, mixed=False)
    host[0]["alpha"], host[0]["beta"] = 0.0, 2.0
    host[0]["A"][:] = np.nan
    host[3]["beta"] = 0.0
    host[3]["C"][:] = np.nan
    host[1]["beta"] = 0.5
    dev, probs = to_device(host)
    assert eb.gemm_grouped("d", probs) == eb.EB2_OK
    torch.cuda.synchronize()
    np.testing.assert_array_equal(back(dev[0][2]), 2.0 * host[0]["C"])   # alpha == 0: A (NaN) not read
    np.testing.assert_array_equal(back(dev[1][2]), 0.5 * host[1]["C"])   # k == 0: beta * C
    assert np.isfinite(back(dev[3][2])[:7, :3]).all()                    # beta == 0: NaN in C discarded


def test_grouped_rejects_bad_problem_with_its_index():
    host = make_batch([(5, 4, 3), (6, 6, 6)], "d", seed=6, mixed=False)
    host[1]["lda"] = 2  # < m
    dev, probs = to_device(host)
    eb.clear_error()
    assert eb.gemm_grouped("d", probs) == eb.EB2_ERR_ARG
    code, msg = eb.last_error()
    assert code == eb.EB2_ERR_ARG and "problem 1" in msg and "info 8" in msg


@pytest.mark.parametrize("dtype", ["d", "s"])
def test_gemm_each_equals_grouped(dtype):
    """The per-product plain launches and the grouped launch produce identical bits."""
    sizes = batch_sizes(120, seed=8)
    host = make_batch(sizes, dtype, seed=9)
    dev1, p1 = to_device(host)
    dev2, p2 = to_device(host)
    assert eb.gemm_grouped(dtype, p1) == eb.EB2_OK
    assert eb.gemm_each(dtype, p2) == eb.EB2_OK
    torch.cuda.synchronize()
    for (a1, b1, c1), (a2, b2, c2) in zip(dev1, dev2):
        assert torch.equal(c1, c2)


@pytest.mark.parametrize("dtype", ["d", "s"])
def test_grouped_classes_give_the_same_bits(dtype):
    """Four products of <= 8 x 8 per warp, two of <= 16 x 16, or every product as 32 x 32
    tiles: each output sees the same operations in the same order."""
    sizes = batch_sizes(200, seed=21, lo=2, hi=40) + [(8, 8, 200), (3, 16, 5), (16, 2, 300), (1, 1, 1), (9, 8, 7)]
    host = make_batch(sizes, dtype, seed=22)
    results = []
    for small, mid in ((8, 16), (0, 0), (8, 0), (0, 16), (4, 12)):
        assert eb.set_grouped_classes(small, mid) == eb.EB2_OK
        dev, probs = to_device(host)
        assert eb.gemm_grouped(dtype, probs) == eb.EB2_OK
        torch.cuda.synchronize()
        results.append([back(c) for (_, _, c) in dev])
    for other in results[1:]:
        for a, b in zip(results[0], other):
            np.testing.assert_array_equal(a, b)
    assert eb.set_grouped_classes(9, 16) == eb.EB2_ERR_ARG


def test_grouped_fp32_no_less_accurate_than_ffma():
    """Normwise error over the batch against the FP64 product of the same FP32 inputs: the
    split-BF16 grouped result against one FFMA SGEMM call per product."""
    sizes = batch_sizes(150, seed=31)
    host = make_batch(sizes, "s", seed=32, mixed=False)
    dev, probs = to_device(host)
    assert eb.gemm_grouped("s", probs) == eb.EB2_OK
    torch.cuda.synchronize()
    eb.set_sgemm_method(eb.METHOD_NATIVE)
    err_g = err_f = norm = 0.0
    for h, (_, _, tC) in zip(host, dev):
        m, n, k = h["m"], h["n"], h["k"]
        A64, B64 = h["A"].astype(np.float64), h["B"].astype(np.float64)
        exact = h["alpha"] * (A64[:m, :k] @ B64[:k, :n])
        ffma = h["C"].copy(order="F")
        eb.sgemm("N", "N", m, n, k, h["alpha"], h["A"], h["lda"], h["B"], h["ldb"], 0.0, ffma, h["ldc"])
        err_g += float(np.sum((back(tC)[:m, :n] - exact) ** 2))
        err_f += float(np.sum((ffma[:m, :n] - exact) ** 2))
        norm += float(np.sum(exact ** 2))
    assert np.sqrt(err_g / norm) <= np.sqrt(err_f / norm), (np.sqrt(err_g / norm), np.sqrt(err_f / norm))
