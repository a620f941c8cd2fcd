"""The configuration picker's MLP: host forward, device forward/backward/Adam kernels,
checked against a float64 numpy restatement of the same network (the checker)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import eigen_b200 as eb

F, H, NC, NS = 8, 64, 12, 7
O = NC + NS


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    o = 0

    def take(*shape):
        nonlocal o
        n = int(np.prod(shape))
        out = w[o:o + n].reshape(shape)
        o += n
        return out

    W1, b1, W2, b2, W3, b3 = take(H, F), take(H), take(H, H), take(H), take(O, H), take(O)
    return W1, b1, W2, b2, W3, b3


def np_forward(w, X):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    h1 = np.maximum(X @ W1.T + b1, 0)
    h2 = np.maximum(h1 @ W2.T + b2, 0)
    return h1, h2, h2 @ W3.T + b3


def np_loss_grad(w, X, yc, ys):
    """Mean over the batch of CE(config logits, yc) + [ys >= 0] CE(slice logits, ys)."""
    W1, b1, W2, b2, W3, b3 = unpack(w)
    h1, h2, out = np_forward(w, X)
    B = X.shape[0]
    g3 = np.zeros_like(out)
    loss = 0.0
    for lo, hi, y, mask in ((0, NC, yc, np.ones(B, bool)), (NC, O, ys, ys >= 0)):
        z = out[:, lo:hi]
        z = z - z.max(1, keepdims=True)
        p = np.exp(z) / np.exp(z).sum(1, keepdims=True)
        idx = np.where(mask)[0]
        loss += -np.log(p[idx, y[idx]]).sum() / B
        gp = p.copy()
        gp[idx, y[idx]] -= 1.0
        gp[~mask] = 0.0
        g3[:, lo:hi] = gp / B
    gW3 = g3.T @ h2
    gb3 = g3.sum(0)
    g2 = (g3 @ W3) * (h2 > 0)
    gW2 = g2.T @ h1
    gb2 = g2.sum(0)
    g1 = (g2 @ W2) * (h1 > 0)
    gW1 = g1.T @ X
    gb1 = g1.sum(0)
    grad = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, grad


def random_weights(seed):
    rng = np.random.default_rng(seed)
    n = eb.load().eb2_mlp_param_count()
    return (rng.standard_normal(n) * 0.3).astype(np.float32)


def test_param_count():
    assert eb.load().eb2_mlp_param_count() == H * F + H + H * H + H + O * H + O


def test_host_forward_matches_numpy():
    lib = eb.load()
    w = random_weights(1)
    rng = np.random.default_rng(2)
    for _ in range(20):
        x = rng.uniform(-1, 1, F).astype(np.float32)
        lg = (ctypes.c_float * O)()
        lib.eb2_picker_forward_host(w.ctypes.data_as(ctypes.c_void_p), x.ctypes.data_as(ctypes.c_void_p), lg)
        ref = np_forward(w.astype(np.float64), x[None, :].astype(np.float64))[2][0]
        np.testing.assert_allclose(np.array(lg), ref, rtol=1e-4, atol=1e-4)


# configuration classes of each kind (blas.h): DGEMM, SGEMM, grouped batch
KINDS = {(b"d", 1): range(0, 6), (b"s", 1): range(6, 10), (b"d", 500): range(10, 12), (b"s", 64): range(10, 12)}


def test_features_and_predict():
    lib = eb.load()
    out = (ctypes.c_float * F)()
    lib.eb2_picker_features(8192, 4096, 1024, b"d", 3.2, 1, 2.0 ** -40, out)
    f = np.array(out)
    np.testing.assert_allclose(f[:4], [13 / 14, 12 / 14, 10 / 14, 1.0], rtol=1e-6)
    assert abs(f[4] - 3.2 / 32) < 1e-6 and f[5] == 0.0
    assert abs(f[6] - 35 / 42) < 1e-6 and abs(f[7] - 40 / 64) < 1e-6
    lib.eb2_picker_features(8, 8, 8, b"s", 0.0, 1024, 0.0, out)  # no target: feature 0
    assert abs(out[5] - 10 / 14) < 1e-6 and out[7] == 0.0
    w = random_weights(3)
    assert eb.set_picker(w) == eb.EB2_OK
    cfg, sl = ctypes.c_int(), ctypes.c_int()
    for (dt, batch), classes in KINDS.items():
        assert lib.eb2_picker_predict(8192, 2048, 700, dt, 1.4, batch, 2.0 ** -45, ctypes.byref(cfg),
                                      ctypes.byref(sl)) == eb.EB2_OK
        x = (ctypes.c_float * F)()
        lib.eb2_picker_features(8192, 2048, 700, dt, 1.4, batch, 2.0 ** -45, x)
        lg = np_forward(w.astype(np.float64), np.array(x, dtype=np.float64)[None, :])[2][0]
        assert cfg.value == max(classes, key=lambda c: lg[c])  # the best class of the call's kind
        assert sl.value == 6 + int(np.argmax(lg[NC:]))
    assert eb.set_picker(np.zeros(5, np.float32)) == eb.EB2_ERR_ARG
    assert eb.set_picker(None) == eb.EB2_OK
    assert lib.eb2_picker_predict(8, 8, 8, b"d", 0.0, 1, 2.0 ** -53, ctypes.byref(cfg),
                                  ctypes.byref(sl)) == eb.EB2_ERR_ARG


def test_set_config_range():
    assert eb.set_config(-1) == eb.EB2_OK
    assert eb.set_config(11) == eb.EB2_OK
    assert eb.set_config(12) == eb.EB2_ERR_ARG
    assert eb.set_config(-2) == eb.EB2_ERR_ARG
    assert eb.load().eb2_config_count() == NC
    assert eb.set_config(-1) == eb.EB2_OK


def test_numpy_gradient_matches_finite_differences():
    """The checker itself: analytic gradient vs central differences (float64)."""
    rng = np.random.default_rng(4)
    w = random_weights(5).astype(np.float64)
    X = rng.uniform(-1, 1, (16, F))
    yc = rng.integers(0, NC, 16)
    ys = rng.integers(-1, NS, 16)
    _, g = np_loss_grad(w, X, yc, ys)
    for i in rng.choice(len(w), 40, replace=False):
        e = np.zeros_like(w)
        e[i] = 1e-6
        fd = (np_loss_grad(w + e, X, yc, ys)[0] - np_loss_grad(w - e, X, yc, ys)[0]) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd)


# ------------------------------------------------------------------ GPU kernels
torch = pytest.importorskip("torch")


def _gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.gpu
def test_device_forward_matches_host_and_numpy():
    _gpu()
    lib = eb.load()
    w = random_weights(6)
    rng = np.random.default_rng(7)
    X = rng.uniform(-1, 1, (300, F)).astype(np.float32)
    dw, dX = torch.from_numpy(w).cuda(), torch.from_numpy(X).cuda()
    dl = torch.empty((300, O), dtype=torch.float32, device="cuda")
    assert lib.eb2_mlp_forward(dw.data_ptr(), dX.data_ptr(), 300, dl.data_ptr(), None) == eb.EB2_OK
    torch.cuda.synchronize()
    got = dl.cpu().numpy()
    ref = np_forward(w.astype(np.float64), X.astype(np.float64))[2]
    np.testing.assert_allclose(got, ref, rtol=1e-4, atol=1e-4)
    for i in range(0, 300, 37):  # host forward: same operations, same float32 results
        lg = (ctypes.c_float * O)()
        lib.eb2_picker_forward_host(w.ctypes.data_as(ctypes.c_void_p), X[i].ctypes.data_as(ctypes.c_void_p), lg)
        np.testing.assert_allclose(np.array(lg), got[i], rtol=1e-6, atol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("batch", [1, 63, 200])
def test_device_gradient_matches_oracle(batch):
    _gpu()
    lib = eb.load()
    rng = np.random.default_rng(batch)
    w = random_weights(batch + 10)
    X = rng.uniform(-1, 1, (batch, F)).astype(np.float32)
    yc = rng.integers(0, NC, batch).astype(np.int32)
    ys = rng.integers(-1, NS, batch).astype(np.int32)
    dw, dX = torch.from_numpy(w).cuda(), torch.from_numpy(X).cuda()
    dyc, dys = torch.from_numpy(yc).cuda(), torch.from_numpy(ys).cuda()
    g = torch.empty_like(dw)
    loss = torch.empty(1, dtype=torch.float32, device="cuda")
    assert lib.eb2_mlp_backward(dw.data_ptr(), dX.data_ptr(), dyc.data_ptr(), dys.data_ptr(), batch, g.data_ptr(),
                                loss.data_ptr(), None) == eb.EB2_OK
    torch.cuda.synchronize()
    ref_loss, ref_g = np_loss_grad(w.astype(np.float64), X.astype(np.float64), yc, ys)
    assert abs(loss.item() - ref_loss) <= 1e-4 * max(1.0, abs(ref_loss))
    got = g.cpu().numpy().astype(np.float64)
    scale = np.abs(ref_g).max()
    assert np.max(np.abs(got - ref_g)) <= 1e-4 * scale + 1e-7


@pytest.mark.gpu
def test_training_kernels_fit_a_separable_problem():
    """Full-batch Adam on the device kernels drives the loss down and classifies a
    synthetic rule (config = which of two features is larger; slices from a third)."""
    _gpu()
    lib = eb.load()
    rng = np.random.default_rng(11)
    X = rng.uniform(0, 1, (512, F)).astype(np.float32)
    yc = np.where(X[:, 0] > X[:, 1], 1, 7).astype(np.int32)
    ys = np.minimum((X[:, 4] * NS).astype(np.int32), NS - 1)
    w = random_weights(12) * 0.5
    dw, dX = torch.from_numpy(w).cuda(), torch.from_numpy(X).cuda()
    dyc, dys = torch.from_numpy(yc).cuda(), torch.from_numpy(ys).cuda()
    g, m1, v1 = torch.zeros_like(dw), torch.zeros_like(dw), torch.zeros_like(dw)
    loss = torch.empty(1, dtype=torch.float32, device="cuda")
    losses = []
    for step in range(1, 1501):
        lib.eb2_mlp_backward(dw.data_ptr(), dX.data_ptr(), dyc.data_ptr(), dys.data_ptr(), 512, g.data_ptr(),
                             loss.data_ptr(), None)
        lib.eb2_mlp_adam(dw.data_ptr(), g.data_ptr(), m1.data_ptr(), v1.data_ptr(), step, 3e-3, None)
        if step in (1, 1500):
            torch.cuda.synchronize()
            losses.append(loss.item())
    assert losses[-1] < 0.25 * losses[0]
    out = np_forward(dw.cpu().numpy().astype(np.float64), X.astype(np.float64))[2]
    assert np.mean(np.argmax(out[:, :NC], 1) == yc) > 0.95
    assert np.mean(np.argmax(out[:, NC:], 1) == ys) > 0.8


# ------------------------------------------------------------------ the trained picker
DATA = eb.LIB_PATH.parent.parent / "data"


def test_trained_picker_beats_the_rules_without_it():
    """On the held-out rows the tuner measured on a B200 (recorded device times of every
    configuration class), the committed weights pick classes whose total time is below the
    library's size rules and close to the exhaustive best, for DGEMM, SGEMM and grouped
    batches; the DGEMM precision label (fewest moduli meeting a swept accuracy target) varies,
    and the predicted count meets it on nearly every row."""
    import json

    from eigen_b200 import tune

    rep = json.loads((DATA / "tune_report.json").read_text())
    raw = (DATA / "picker_weights.bin").read_bytes()
    assert raw[:8] == b"EB2PICK1"
    count = int.from_bytes(raw[8:12], "little")
    w = np.frombuffer(raw[16:16 + 4 * count], dtype="<f4").astype(np.float32)
    assert count == eb.load().eb2_mlp_param_count()
    summary, rows = tune.compare(rep["holdout_rows"], w, rep["device"]["sms"])
    assert summary["n"] >= 400
    assert summary["total_ms_picker"] < 0.9 * summary["total_ms_default"]
    assert summary["total_ms_picker"] < 1.1 * summary["total_ms_best"]
    for kind in ("d", "s", "b"):
        k = summary["per_kind"][kind]
        assert k["n"] >= 20, kind
        assert k["total_ms_picker"] <= 1.02 * k["total_ms_default"], (kind, k)
    d = summary["per_kind"]["d"]
    assert len(d["moduli_label_counts"]) >= 3  # a label with variance
    assert d["moduli_pass_rate"] >= 0.9
