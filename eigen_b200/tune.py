"""Autotuner and learned configuration picker for the DGEMM path.

The counterpart of Eigen's blocking-size heuristic
(Eigen/src/Core/products/GeneralBlockPanelKernel.h:202-452, computeProductBlockingSizes):
instead of a cache model, an exhaustive autotuner times every kernel configuration on
random shapes and a small MLP learns to predict the best one, plus the number of CRT
moduli the emulated DGEMM needs to meet its accuracy target.

    python -m eigen_b200.tune all [--train 2000] [--holdout 500] [--out eigen_b200/data]

* collect : for each shape (m, n, k log-uniform in [3, max-dim]; entries u*2^e with e in
            [-r, r], r uniform in 0..32) the modulus count the a-posteriori check settles
            on (starting from 8, two at a time), then the device time of every
            configuration at that count: native FP64 kernel; CRT emulation with one CTA
            per 128 x 256 tile; CRT emulation with a CTA pair per 256 x 256 tile.
* train   : the MLP (eb2_mlp_param_count() weights) is trained on the GPU by the
            library's own CUDA kernels (eb2_mlp_backward / eb2_mlp_adam), full batch,
            cross-entropy on the best configuration and on the precision class
            c = (moduli - 8) / 2.
* evaluate: on held-out shapes, regret of the picked configuration against the
            exhaustive best, next to the regret of the library's rule without a picker
            (native below ~2^32 multiply-adds, else CRT, pair tiles when they fill the
            SMs, 16 moduli plus escalation).
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

CONFIGS = [0, 256, 512]  # 0 = native; CRT with one CTA per 128 x 256 tile; CRT with CTA pairs (256 x 256)
SLICE_BASE, NUM_SLICES = 6, 7  # the picker's precision head: class c -> 8 + 2c moduli
MODULI_MIN, MODULI_MAX = 8, 20
PICKER_MAGIC = b"EB2PICK1"


def shapes(count, seed, lo=3, hi=16384):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        m, n, k = (int(round(math.exp(rng.uniform(math.log(lo), math.log(hi))))) for _ in range(3))
        r = int(rng.integers(0, 33))
        out.append(dict(m=m, n=n, k=k, dtype="d", r=r))
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


def _reset():
    eb.set_dgemm_method(eb.METHOD_AUTO)
    eb.set_tile_n(0)
    eb.set_dgemm_moduli(0)
    eb.set_dgemm_tolerance(2.0 ** -53)


def measure_shape(torch, pool, sh, gen, reps=3):
    m, n, k, dt, r = sh["m"], sh["n"], sh["k"], sh["dtype"], sh["r"]
    A, B, C = pool.get(dt)
    a = fill(torch, A, m, k, r, gen)
    b = fill(torch, B, k, n, r, gen)
    c = C[: m * n]
    rec = dict(sh, spread=0.0)
    eb.set_picker(None)
    # modulus count the a-posteriori check settles on for this data (from 8, two at a time)
    eb.set_dgemm_method(eb.METHOD_CRT)
    eb.set_dgemm_moduli(MODULI_MIN)
    eb.set_dgemm_tolerance(2.0 ** -53)
    rc = eb.dgemm_device("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, c, m, check_accuracy=True)
    info = eb.last_call_info()
    rec["spread"] = float(info["spread"])
    need = info["slices"] if rc == eb.EB2_OK else MODULI_MAX
    rec["moduli"] = int(min(max(need, MODULI_MIN), MODULI_MAX))
    eb.set_dgemm_moduli(rec["moduli"])
    eb.set_dgemm_tolerance(1.0)  # time exactly that many moduli
    times = {}
    for cfg in CONFIGS:
        if cfg == 0:
            eb.set_dgemm_method(eb.METHOD_NATIVE)
        else:
            eb.set_dgemm_method(eb.METHOD_CRT)
            eb.set_tile_n(cfg)
        fn = lambda: eb.dgemm_device("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, c, m, check_accuracy=True)
        times[str(cfg)] = time_call(torch, fn, reps)
    rec["times_ms"] = times
    rec["best"] = int(min(times, key=lambda c: times[c]))
    _reset()
    return rec


def features(sh, spread=None):
    """The feature vector the library computes for this call (spread: the scan's
    exponent-spread statistic, as measured on the shape's data; 0 for SGEMM)."""
    out = (ctypes.c_float * 8)()
    sp = sh.get("spread", 0.0) if spread is None else spread
    eb.load().eb2_picker_features(sh["m"], sh["n"], sh["k"], sh["dtype"].encode(), sp, 1, out)
    return list(out)


def labels(rec):
    cfg_index = {0: 0, 256: 1, 512: 2}[rec["best"]]
    return cfg_index, (rec["moduli"] - MODULI_MIN) // 2


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
    """(configuration, moduli) the library picks with weights w; configuration 3 (the
    digit-slice scheme) and a native pick are both reported as 0 / native."""
    lib = eb.load()
    x = (ctypes.c_float * 8)(*features(sh, spread))
    lg = (ctypes.c_float * 11)()
    wa = w.ctypes.data_as(ctypes.c_void_p)
    lib.eb2_picker_forward_host(wa, x, lg)
    lg = list(lg)
    cfg = int(np.argmax(lg[:4]))
    moduli = MODULI_MIN + 2 * int(np.argmax(lg[4:]))
    return {1: 256, 2: 512}.get(cfg, 0), moduli


def default_choice(sh, num_sms):
    """What the library does without a picker (gemm_driver.cpp): native below ~2^32
    multiply-adds, thin k or thin m/n; else CRT, CTA pairs when they fill the SMs, 16 moduli."""
    m, n, k = sh["m"], sh["n"], sh["k"]
    if not (m * n * k >= 2 ** 32 and k >= 1024 and min(m, n) >= 256):
        return 0, 16
    pair_tiles = ((m + 255) // 256) * ((n + 255) // 256)
    return (512 if 2 * pair_tiles >= num_sms else 256), 16


def charged_time(rec, cfg, moduli):
    """Device time of configuration `cfg` run with `moduli` moduli, from the measured time
    at the needed count: fewer than needed costs one more full pass per escalation (two
    moduli each), more than needed scales with the modulus count."""
    t = rec["times_ms"][str(cfg)]
    if cfg == 0:
        return t
    need = rec["moduli"]
    if moduli >= need:
        return t * moduli / need
    passes = (need - moduli + 1) // 2
    return t * (1.0 + sum((moduli + 2 * i) / need for i in range(passes)))


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


def compare(rows, w, num_sms):
    """Regret (time / exhaustive best - 1) of the picker and of the no-picker rule on
    measured rows; pure host computation on recorded times."""
    out = []
    for rec in rows:
        best = rec["times_ms"][str(rec["best"])]
        pc, pm = predict(w, rec)
        dc, dm = default_choice(rec, num_sms)
        out.append(dict(m=rec["m"], n=rec["n"], k=rec["k"], r=rec["r"], best=rec["best"], moduli=rec["moduli"],
                        pick_cfg=pc, pick_moduli=pm, default_cfg=dc,
                        regret_picker=charged_time(rec, pc, pm) / best - 1.0,
                        regret_default=charged_time(rec, dc, dm) / best - 1.0,
                        t_best=best, t_picker=charged_time(rec, pc, pm), t_default=charged_time(rec, dc, dm)))
    rp = np.array([o["regret_picker"] for o in out])
    rd = np.array([o["regret_default"] for o in out])
    summary = dict(n=len(out), regret_mean=float(rp.mean()), regret_p50=float(np.median(rp)),
                   regret_p95=float(np.percentile(rp, 95)), default_regret_mean=float(rd.mean()),
                   default_regret_p95=float(np.percentile(rd, 95)),
                   total_ms_best=float(sum(o["t_best"] for o in out)),
                   total_ms_picker=float(sum(o["t_picker"] for o in out)),
                   total_ms_default=float(sum(o["t_default"] for o in out)),
                   exact_best=float(np.mean([o["pick_cfg"] == o["best"] for o in out])),
                   moduli_pass_rate=float(np.mean([o["pick_moduli"] >= o["moduli"] for o in out])))
    return summary, out


def evaluate(torch, pool, w, held, gen, num_sms):
    rows = [measure_shape(torch, pool, sh, gen, reps=2) for sh in held]
    summary, _ = compare(rows, w, num_sms)
    return summary, rows


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
    summary, rows = evaluate(torch, pool, w, held, gen, key["sms"])
    report = dict(device=key, train=len(db), holdout=len(held), max_dim=md, loss_history=hist, **summary,
                  seconds=round(time.time() - t0, 1))
    (out / "tune_report.json").write_text(json.dumps(dict(report, holdout_rows=rows)))
    print(json.dumps(report))
    return 0


if __name__ == "__main__":
    sys.exit(main())
