"""Autotuner and learned configuration picker for the emulated products.

The counterpart of Eigen's blocking-size heuristic
(Eigen/src/Core/products/GeneralBlockPanelKernel.h:202-452, computeProductBlockingSizes):
instead of a cache model, an exhaustive autotuner times every kernel configuration on
random shapes and a small MLP learns to predict the best one, plus the digit-slice count
the emulated DGEMM needs to meet its accuracy target.

    python -m eigen_b200.tune all [--train 2000] [--holdout 500] [--out eigen_b200/data]

* collect : for each shape (m, n, k log-uniform in [3, 16384]; dtype f64 or f32; entries
            u*2^e with e in [-r, r], r uniform in 0..32) the slice count the a-posteriori
            check settles on (f64), then the device time of every configuration
            (native; emulated 128x128, 128x256, CTA pair) at that slice count.
* train   : the MLP (eb2_mlp_param_count() weights) is trained on the GPU by the
            library's own CUDA kernels (eb2_mlp_backward / eb2_mlp_adam), full batch,
            cross-entropy on the best configuration and on the needed slice count.
* evaluate: on held-out shapes, regret of the picked configuration against the
            exhaustive best, how often the picked slice count meets the target without
            escalation, and the same call timed with and without the picker.
Outputs: <out>/tune_db.json, <out>/picker_weights.bin (+ .json metadata), <out>/tune_report.json.
The library reads picker_weights.bin next to itself (eigen_b200/data) when the GPU matches.
"""
from __future__ import annotations

import argparse
import ctypes
import hashlib
import json
import math
import struct
import sys
import time
from pathlib import Path

import numpy as np

import eigen_b200 as eb

CONFIGS = [0, 128, 256, 512]  # 0 = native; tile configurations of the emulated products
SLICE_BASE, NUM_SLICES = 6, 7
PICKER_MAGIC = b"EB2PICK1"


def shapes(count, seed, lo=3, hi=16384):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        m, n, k = (int(round(math.exp(rng.uniform(math.log(lo), math.log(hi))))) for _ in range(3))
        dtype = "d" if rng.random() < 0.6 else "s"
        r = int(rng.integers(0, 33))
        out.append(dict(m=m, n=n, k=k, dtype=dtype, r=r))
    return out


class Pool:
    """Device buffers reused across shapes (column-major views with ld = rows)."""

    def __init__(self, torch, max_elems_a, max_elems_b, max_elems_c):
        self.torch = torch
        self.cap = (max_elems_a, max_elems_b, max_elems_c)
        self.bufs = {}

    def get(self, dtype):
        t = self.torch
        tdt = t.float64 if dtype == "d" else t.float32
        if dtype not in self.bufs:
            self.bufs[dtype] = [t.empty(c, dtype=tdt, device="cuda") for c in self.cap]
        return self.bufs[dtype]


def fill(torch, buf, rows, cols, r, gen):
    n = rows * cols
    x = buf[:n]
    x.uniform_(-1.0, 1.0, generator=gen)
    if r:
        e = torch.randint(-r, r + 1, (n,), device="cuda", generator=gen).to(x.dtype)
        x.mul_(torch.exp2(e))
    return x


def time_call(torch, fn, reps=3):
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fn()
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(reps):
        ev0.record()
        fn()
        ev1.record()
        torch.cuda.synchronize()
        best = min(best, ev0.elapsed_time(ev1))
    return best


def measure_shape(torch, pool, sh, gen, reps=3):
    m, n, k, dt, r = sh["m"], sh["n"], sh["k"], sh["dtype"], sh["r"]
    A, B, C = pool.get(dt)
    a = fill(torch, A, m, k, r, gen)
    b = fill(torch, B, k, n, r, gen)
    c = C[: m * n]
    rec = dict(sh, spread=0.0)
    eb.set_picker(None)
    if dt == "d":
        # slice count the a-posteriori check settles on for this data
        eb.set_dgemm_method(eb.METHOD_EMULATED)
        eb.set_tile_n(128)
        eb.set_dgemm_slices(SLICE_BASE)
        eb.set_dgemm_tolerance(2.0 ** -53)
        rc = eb.dgemm_device("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, c, m, check_accuracy=True)
        info = eb.last_call_info()
        rec["spread"] = float(info["spread"])
        need = info["slices"] if rc == eb.EB2_OK else SLICE_BASE + NUM_SLICES - 1
        rec["slices"] = int(min(max(need, SLICE_BASE), SLICE_BASE + NUM_SLICES - 1))
        eb.set_dgemm_slices(rec["slices"])
        eb.set_dgemm_tolerance(1.0)  # time exactly that many slices
    times = {}
    for cfg in CONFIGS:
        if dt == "d" and cfg == 256:
            continue  # the Ozaki GEMM has no 128x256 single-CTA tile (256 selects the pair)
        if cfg == 0:
            if dt == "d":
                eb.set_dgemm_method(eb.METHOD_NATIVE)
            else:
                eb.set_sgemm_method(eb.METHOD_NATIVE)
        else:
            eb.set_tile_n(cfg)
            if dt == "d":
                eb.set_dgemm_method(eb.METHOD_EMULATED)
            else:
                eb.set_sgemm_method(eb.METHOD_EMULATED)
        if dt == "d":
            fn = lambda: eb.dgemm_device("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, c, m, check_accuracy=True)
        else:
            fn = lambda: eb.sgemm_device("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, c, m)
        times[str(cfg)] = time_call(torch, fn, reps)
    rec["times_ms"] = times
    rec["best"] = int(min(times, key=lambda c: times[c]))
    eb.set_dgemm_method(eb.METHOD_AUTO)
    eb.set_sgemm_method(eb.METHOD_AUTO)
    eb.set_tile_n(0)
    eb.set_dgemm_slices(0)
    eb.set_dgemm_tolerance(2.0 ** -53)
    return rec


def features(sh, spread=None):
    """The feature vector the library computes for this call (spread: the scan's
    exponent-spread statistic, as measured on the shape's data; 0 for SGEMM)."""
    out = (ctypes.c_float * 8)()
    sp = sh.get("spread", 0.0) if spread is None else spread
    eb.load().eb2_picker_features(sh["m"], sh["n"], sh["k"], sh["dtype"].encode(), sp, 1, out)
    return list(out)


def labels(rec):
    cfg_index = {0: 0, 128: 1, 256: 2, 512: 3}[rec["best"]]
    sl = rec["slices"] - SLICE_BASE if rec["dtype"] == "d" else -1
    return cfg_index, sl


def train(torch, db, steps=4000, lr=3e-3, seed=0):
    lib = eb.load()
    n_params = lib.eb2_mlp_param_count()
    X = torch.tensor([features(r) for r in db], dtype=torch.float32, device="cuda")
    lab = [labels(r) for r in db]
    yc = torch.tensor([c for c, _ in lab], dtype=torch.int32, device="cuda")
    ys = torch.tensor([s for _, s in lab], dtype=torch.int32, device="cuda")
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    w = torch.empty(n_params, dtype=torch.float32, device="cuda")
    # He-style init, layer by layer (W1[64][8] b1 W2[64][64] b2 W3[11][64] b3)
    sizes = [(64, 8), (64,), (64, 64), (64,), (11, 64), (11,)]
    off = 0
    for s in sizes:
        cnt = int(np.prod(s))
        if len(s) == 2:
            w[off:off + cnt].normal_(0.0, math.sqrt(2.0 / s[1]), generator=g)
        else:
            w[off:off + cnt].zero_()
        off += cnt
    grads = torch.zeros_like(w)
    m1 = torch.zeros_like(w)
    v1 = torch.zeros_like(w)
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    hist = []
    for step in range(1, steps + 1):
        lib.eb2_mlp_backward(w.data_ptr(), X.data_ptr(), yc.data_ptr(), ys.data_ptr(), len(db), grads.data_ptr(),
                             loss.data_ptr(), None)
        lib.eb2_mlp_adam(w.data_ptr(), grads.data_ptr(), m1.data_ptr(), v1.data_ptr(), step, lr, None)
        if step % 500 == 0 or step == 1:
            torch.cuda.synchronize()
            hist.append((step, float(loss.item())))
    torch.cuda.synchronize()
    return w.cpu().numpy().astype(np.float32), hist


def predict(w, sh, spread=None):
    lib = eb.load()
    x = (ctypes.c_float * 8)(*features(sh, spread))
    lg = (ctypes.c_float * 11)()
    wa = w.ctypes.data_as(ctypes.c_void_p)
    lib.eb2_picker_forward_host(wa, x, lg)
    lg = list(lg)
    cfg = int(np.argmax(lg[:4]))
    s = SLICE_BASE + int(np.argmax(lg[4:]))
    return [0, 128, 256, 512][cfg], s


def device_key(torch):
    p = torch.cuda.get_device_properties(0)
    return dict(name=p.name, sms=p.multi_processor_count, cc=f"{p.major}.{p.minor}")


def write_weights(path: Path, w: np.ndarray, key: dict):
    """picker_weights.bin: magic, uint32 count, uint32 SM count, then count float32."""
    path.parent.mkdir(parents=True, exist_ok=True)
    with open(path, "wb") as f:
        f.write(PICKER_MAGIC)
        f.write(struct.pack("<II", len(w), key["sms"]))
        f.write(w.astype("<f4").tobytes())
    meta = dict(key, count=int(len(w)), sha256=hashlib.sha256(w.tobytes()).hexdigest(),
                build=hashlib.sha256(eb.LIB_PATH.read_bytes()).hexdigest()[:16])
    path.with_suffix(".json").write_text(json.dumps(meta, indent=1))


def evaluate(torch, pool, w, held, gen):
    rows = []
    for sh in held:
        rec = measure_shape(torch, pool, sh, gen, reps=2)
        cfg, s = predict(w, rec)
        t_best = rec["times_ms"][str(rec["best"])]
        key = str(cfg if not (sh["dtype"] == "d" and cfg == 256) else 512)
        t_pick = rec["times_ms"].get(key, float("nan"))
        ok_slices = (sh["dtype"] == "s") or (s >= rec["slices"])
        # a slice count below the need costs an escalation pass: charge the exhaustive
        # time of the chosen configuration scaled by the extra diagonal's work
        if sh["dtype"] == "d" and cfg != 0 and s < rec["slices"]:
            t_pick *= 1.0 + (rec["slices"] - s) * (rec["slices"] + 1) / (rec["slices"] * (rec["slices"] + 1) / 2)
        rows.append(dict(rec, pick_cfg=cfg, pick_slices=s, regret=t_pick / t_best - 1.0, slices_ok=ok_slices))
    reg = np.array([r["regret"] for r in rows])
    return dict(n=len(rows), regret_mean=float(np.nanmean(reg)), regret_p50=float(np.nanmedian(reg)),
                regret_p95=float(np.nanpercentile(reg, 95)),
                exact_best=float(np.mean([r["pick_cfg"] == r["best"] or
                                          (r["dtype"] == "d" and r["pick_cfg"] == 256 and r["best"] == 512)
                                          for r in rows])),
                slice_pass_rate=float(np.mean([r["slices_ok"] for r in rows if r["dtype"] == "d"] or [1.0]))), rows


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("cmd", choices=["all"])
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--holdout", type=int, default=500)
    ap.add_argument("--max-dim", type=int, default=16384)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--out", default=str(Path(__file__).resolve().parent / "data"))
    a = ap.parse_args(argv)
    import torch

    out = Path(a.out)
    out.mkdir(parents=True, exist_ok=True)
    eb.load()
    md = a.max_dim
    pool = Pool(torch, md * md, md * md, md * md)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(123)
    t0 = time.time()
    train_shapes = shapes(a.train, seed=1, hi=md)
    db = []
    for i, sh in enumerate(train_shapes):
        db.append(measure_shape(torch, pool, sh, gen))
        if (i + 1) % 250 == 0:
            print(f"collected {i + 1}/{len(train_shapes)} in {time.time() - t0:.0f}s", flush=True)
    key = device_key(torch)
    (out / "tune_db.json").write_text(json.dumps(dict(device=key, shapes=db)))
    w, hist = train(torch, db, steps=a.steps)
    write_weights(out / "picker_weights.bin", w, key)
    held = shapes(a.holdout, seed=2, hi=md)
    summary, rows = evaluate(torch, pool, w, held, gen)
    report = dict(device=key, train=len(db), holdout=len(held), loss_history=hist, **summary,
                  seconds=round(time.time() - t0, 1))
    (out / "tune_report.json").write_text(json.dumps(dict(report, rows=rows)))
    print(json.dumps(report))
    return 0


if __name__ == "__main__":
    sys.exit(main())
