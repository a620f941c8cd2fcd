"""Autotuner and learned configuration picker.

The counterpart of Eigen's blocking-size heuristic
(Eigen/src/Core/products/GeneralBlockPanelKernel.h:202-452, computeProductBlockingSizes):
instead of a cache model, an exhaustive autotuner times every configuration class on random
problems and a small MLP learns to predict the best one, plus the number of CRT moduli the
emulated DGEMM needs to meet an accuracy target.

    python -m eigen_b200.tune all [--train 2000] [--holdout 500] [--out eigen_b200/data]

* collect : rows of three kinds, each timed through the library's entry points with every
            configuration class of its kind forced in turn (eb2_set_config):
            - DGEMM (m, n, k log-uniform in [3, max-dim]; entries u*2^e with e in [-r, r], r
              uniform in 0..32; accuracy target 2^-t, t uniform in [30, 53]): the modulus
              count the a-posteriori check settles on for that target (from 8, two at a
              time), then classes 0-5 at that count: native FP64; CRT one CTA or CTA pair,
              column-major or in raster groups; CRT one CTA with split K;
            - SGEMM (same shapes and data law): classes 6-9: FP32 FFMA; split-BF16 on
              128x128, 128x256 and 256x256 (pair) tiles;
            - grouped batches (count log-uniform in [32, 20000], sizes log-uniform in [3, hi]
              with hi log-uniform in [16, 256], a random share of {3,4,6,8} cubes; FP64 and
              FP32): classes 10-11: size classes 8 / 16, or 32 x 32 tiles only.
* train   : the MLP (eb2_mlp_param_count() weights) is trained on the GPU by the library's
            own CUDA kernels (eb2_mlp_backward / eb2_mlp_adam), full batch, cross-entropy on
            the best class and, for DGEMM rows, on the precision class c = (moduli - 8) / 2.
* evaluate: on held-out rows, the regret of the picked class against the exhaustive best,
            per kind, next to the regret of the library's rules without a picker, and the
            share of DGEMM rows whose predicted modulus count meets the target.
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

# configuration classes (blas.h, eb2_set_config)
D_CONFIGS = [0, 1, 2, 3, 4, 5]
S_CONFIGS = [6, 7, 8, 9]
B_CONFIGS = [10, 11]
NUM_CONFIGS = 12
SLICE_BASE, NUM_SLICES = 6, 7  # the precision head: class c -> 8 + 2c moduli
MODULI_MIN, MODULI_MAX = 8, 20
NUM_OUT = NUM_CONFIGS + NUM_SLICES
PICKER_MAGIC = b"EB2PICK1"
U64, U32 = 2.0 ** -53, 2.0 ** -24


def kind_configs(kind):
    return {"d": D_CONFIGS, "s": S_CONFIGS, "b": B_CONFIGS}[kind]


def shapes(count, seed, lo=3, hi=16384, sgemm_share=0.35):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        m, n, k = (int(round(math.exp(rng.uniform(math.log(lo), math.log(hi))))) for _ in range(3))
        r = int(rng.integers(0, 33))
        if rng.random() < sgemm_share:
            out.append(dict(kind="s", m=m, n=n, k=k, dtype="s", r=r, tol=U32))
        else:
            out.append(dict(kind="d", m=m, n=n, k=k, dtype="d", r=r, tol=2.0 ** -float(rng.uniform(30.0, 53.0))))
    return out


def batches(count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n_prob = int(round(math.exp(rng.uniform(math.log(32), math.log(20000)))))
        hi = float(math.exp(rng.uniform(math.log(16), math.log(256))))
        fixed = float(rng.uniform(0.0, 0.5))
        dtype = "d" if rng.random() < 0.5 else "s"
        out.append(dict(kind="b", dtype=dtype, count=n_prob, hi=hi, fixed=fixed, seed=int(rng.integers(1 << 30)),
                        tol=U64 if dtype == "d" else U32))
    return out


def batch_sizes(b):
    rng = np.random.default_rng(b["seed"])
    sz = []
    for _ in range(b["count"]):
        if rng.random() < b["fixed"]:
            s = int(rng.choice([3, 4, 6, 8]))
            sz.append((s, s, s))
        else:
            sz.append(tuple(int(round(math.exp(rng.uniform(math.log(3.0), math.log(b["hi"]))))) for _ in range(3)))
    return sz


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
    eb.set_config(-1)
    eb.set_dgemm_method(eb.METHOD_AUTO)
    eb.set_sgemm_method(eb.METHOD_AUTO)
    eb.set_tile_n(0)
    eb.set_dgemm_moduli(0)
    eb.set_dgemm_tolerance(2.0 ** -53)
    eb.set_grouped_classes(-1, -1)


def measure_shape(torch, pool, sh, gen, reps=3):
    m, n, k, dt, r = sh["m"], sh["n"], sh["k"], sh["dtype"], sh["r"]
    A, B, C = pool.get(dt)
    a = fill(torch, A, m, k, r, gen)
    b = fill(torch, B, k, n, r, gen)
    c = C[: m * n]
    rec = dict(sh, spread=0.0)
    eb.set_picker(None)
    if dt == "d":
        # modulus count the a-posteriori check settles on for this data and target (from 8, two at a time)
        eb.set_config(1)
        eb.set_dgemm_moduli(MODULI_MIN)
        eb.set_dgemm_tolerance(sh["tol"])
        rc = eb.dgemm_device("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, c, m, check_accuracy=True)
        info = eb.last_call_info()
        rec["spread"] = float(info["spread"])
        need = info["slices"] if rc == eb.EB2_OK else MODULI_MAX
        rec["moduli"] = int(min(max(need, MODULI_MIN), MODULI_MAX))
        eb.set_dgemm_moduli(rec["moduli"])
        eb.set_dgemm_tolerance(1.0)  # time exactly that many moduli
        fn = lambda: eb.dgemm_device("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, c, m, check_accuracy=True)
    else:
        fn = lambda: eb.sgemm_device("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, c, m)
    times, splits = {}, {}
    for cfg in kind_configs(sh["kind"]):
        eb.set_config(cfg)
        times[str(cfg)] = time_call(torch, fn, reps)
        splits[str(cfg)] = int(eb.last_call_info()["splits"])
    rec["times_ms"] = times
    rec["splits"] = splits
    rec["best"] = int(min(times, key=lambda q: times[q]))
    _reset()
    return rec


def measure_batch(torch, bt, reps=3):
    """Device time of one grouped launch of the batch with each size-class configuration."""
    sizes = batch_sizes(bt)
    tdt = torch.float64 if bt["dtype"] == "d" else torch.float32
    na = sum(m * k for m, n, k in sizes)
    nb = sum(k * n for m, n, k in sizes)
    nc = sum(m * n for m, n, k in sizes)
    g = torch.Generator(device="cuda")
    g.manual_seed(bt["seed"])
    bufA = torch.rand(na + 2 * len(sizes), dtype=tdt, device="cuda", generator=g) * 2 - 1
    bufB = torch.rand(nb + 2 * len(sizes), dtype=tdt, device="cuda", generator=g) * 2 - 1
    bufC = torch.zeros(nc + 2 * len(sizes), dtype=tdt, device="cuda")
    es = bufA.element_size()
    probs = []
    oa = ob = oc = 0
    for (m, n, k) in sizes:
        probs.append(dict(m=m, n=n, k=k, alpha=1.0, beta=0.0, a=bufA.data_ptr() + oa * es, lda=m,
                          b=bufB.data_ptr() + ob * es, ldb=k, c=bufC.data_ptr() + oc * es, ldc=m))
        oa += m * k + (m * k) % 2
        ob += k * n + (k * n) % 2
        oc += m * n + (m * n) % 2
    arr = eb.problems_array(probs)
    rec = dict(bt)
    lm = float(np.mean([math.log(m) for m, n, k in sizes]))
    ln = float(np.mean([math.log(n) for m, n, k in sizes]))
    lk = float(np.mean([math.log(k) for m, n, k in sizes]))
    rec.update(m=int(round(math.exp(lm))), n=int(round(math.exp(ln))), k=int(round(math.exp(lk))), spread=0.0)
    times = {}
    for cfg in B_CONFIGS:
        eb.set_config(cfg)
        plan = eb.GroupedPlan(bt["dtype"], arr)
        times[str(cfg)] = time_call(torch, lambda: plan.execute(), reps)
        plan.close()
    _reset()
    rec["times_ms"] = times
    rec["best"] = int(min(times, key=lambda q: times[q]))
    del bufA, bufB, bufC
    return rec


def features(sh, spread=None):
    """The feature vector the library computes for this call (spread: the scan's
    exponent-spread statistic, as measured on the shape's data; 0 for SGEMM and batches)."""
    out = (ctypes.c_float * 8)()
    sp = sh.get("spread", 0.0) if spread is None else spread
    eb.load().eb2_picker_features(sh["m"], sh["n"], sh["k"], sh["dtype"].encode(), sp,
                                  sh["count"] if sh["kind"] == "b" else 1, sh["tol"], out)
    return list(out)


def labels(rec):
    slice_label = (rec["moduli"] - MODULI_MIN) // 2 if rec["kind"] == "d" else -1
    return rec["best"], slice_label


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
    # He-style init, layer by layer (W1[64][8] b1 W2[64][64] b2 W3[19][64] b3)
    sizes = [(64, 8), (64,), (64, 64), (64,), (NUM_OUT, 64), (NUM_OUT,)]
    off = 0
    for s in sizes:
        cnt = int(np.prod(s))
        if len(s) == 2:
            w[off:off + cnt].normal_(0.0, math.sqrt(2.0 / s[1]), generator=g)
        else:
            w[off:off + cnt].zero_()
        off += cnt
    assert off == n_params
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


def _logits(w, sh, spread=None):
    lib = eb.load()
    x = (ctypes.c_float * 8)(*features(sh, spread))
    lg = (ctypes.c_float * NUM_OUT)()
    lib.eb2_picker_forward_host(w.ctypes.data_as(ctypes.c_void_p), x, lg)
    return list(lg)


def predict(w, sh):
    """(configuration class, moduli) the library settles on with weights w: a DGEMM first picks
    native or CRT on the shape alone, then (CRT) the class and the modulus count with the
    scan's spread; SGEMM and batches pick once.  A CRT call whose second prediction is not a CRT
    class keeps the size rule's tile (reported as class 1 or 2 by default_choice's rule)."""
    cfgs = kind_configs(sh["kind"])
    lg = _logits(w, sh, spread=0.0)
    cfg = max(cfgs, key=lambda c: lg[c])
    moduli = 16
    if sh["kind"] == "d" and cfg != 0:
        lg2 = _logits(w, sh)
        moduli = MODULI_MIN + 2 * int(np.argmax(lg2[NUM_CONFIGS:]))
        c2 = max(cfgs, key=lambda c: lg2[c])
        cfg = c2 if c2 != 0 else rule_crt_config(sh)
    return cfg, moduli


def rule_crt_config(sh, num_sms=148):
    pair_tiles = ((sh["m"] + 255) // 256) * ((sh["n"] + 255) // 256)
    return 2 if 2 * pair_tiles >= num_sms else 1


def default_choice(sh, num_sms):
    """What the library does without a picker (gemm_driver.cpp, grouped_api.cpp): DGEMM native
    below ~2^32 multiply-adds, thin k or thin m/n, else CRT (pairs when they fill the SMs) with
    16 moduli; SGEMM split-BF16 on the size rule's tile; batches with size classes 8 / 16."""
    if sh["kind"] == "b":
        return 10, 16
    m, n, k = sh["m"], sh["n"], sh["k"]
    if sh["kind"] == "s":
        if n <= 128:
            return 7, 16
        return (7 if ((m + 127) // 128) * ((n + 255) // 256) < num_sms else 8), 16
    if not (m * n * k >= 2 ** 32 and k >= 1024 and min(m, n) >= 256):
        return 0, 16
    return rule_crt_config(sh, num_sms), 16


def charged_time(rec, cfg, moduli):
    """Device time of class `cfg` with `moduli` moduli, from the measured time at the needed
    count: fewer than needed costs one more full pass per escalation (two moduli each), more
    than needed scales with the modulus count (DGEMM CRT classes only)."""
    t = rec["times_ms"][str(cfg)]
    if rec["kind"] != "d" or cfg == 0:
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
    """Regret (time / exhaustive best - 1) of the picker and of the rules without it on
    measured rows, overall and per kind; pure host computation on recorded times."""
    out = []
    for rec in rows:
        best = rec["times_ms"][str(rec["best"])]
        pc, pm = predict(w, rec)
        dc, dm = default_choice(rec, num_sms)
        o = dict(kind=rec["kind"], m=rec["m"], n=rec["n"], k=rec["k"], best=rec["best"], pick_cfg=pc,
                 pick_moduli=pm, default_cfg=dc, regret_picker=charged_time(rec, pc, pm) / best - 1.0,
                 regret_default=charged_time(rec, dc, dm) / best - 1.0, t_best=best,
                 t_picker=charged_time(rec, pc, pm), t_default=charged_time(rec, dc, dm))
        if rec["kind"] == "d":
            o["moduli"] = rec["moduli"]
        out.append(o)

    def summarize(sel):
        if not sel:
            return dict(n=0)
        rp = np.array([o["regret_picker"] for o in sel])
        rd = np.array([o["regret_default"] for o in sel])
        res = dict(n=len(sel), regret_mean=float(rp.mean()), regret_p50=float(np.median(rp)),
                   regret_p95=float(np.percentile(rp, 95)), default_regret_mean=float(rd.mean()),
                   default_regret_p95=float(np.percentile(rd, 95)),
                   total_ms_best=float(sum(o["t_best"] for o in sel)),
                   total_ms_picker=float(sum(o["t_picker"] for o in sel)),
                   total_ms_default=float(sum(o["t_default"] for o in sel)),
                   exact_best=float(np.mean([o["pick_cfg"] == o["best"] for o in sel])))
        d = [o for o in sel if o["kind"] == "d"]
        if d:
            res["moduli_pass_rate"] = float(np.mean([o["pick_moduli"] >= o["moduli"] for o in d]))
            res["moduli_exact_rate"] = float(np.mean([o["pick_moduli"] == o["moduli"] for o in d]))
            res["moduli_label_counts"] = {str(v): int(c) for v, c in zip(*np.unique([o["moduli"] for o in d],
                                                                                    return_counts=True))}
        return res

    summary = summarize(out)
    summary["per_kind"] = {kd: summarize([o for o in out if o["kind"] == kd]) for kd in ("d", "s", "b")}
    return summary, out


def evaluate(torch, pool, w, held, held_b, gen, num_sms):
    rows = [measure_shape(torch, pool, sh, gen, reps=2) for sh in held]
    rows += [measure_batch(torch, bt, reps=2) for bt in held_b]
    summary, _ = compare(rows, w, num_sms)
    return summary, rows


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("cmd", choices=["all"])
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--holdout", type=int, default=500)
    ap.add_argument("--batches", type=int, default=160, help="grouped-batch rows for training")
    ap.add_argument("--holdout-batches", type=int, default=40)
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
    db = []
    for i, sh in enumerate(shapes(a.train, seed=1, hi=md)):
        db.append(measure_shape(torch, pool, sh, gen))
        if (i + 1) % 250 == 0:
            print(f"collected {i + 1}/{a.train} shapes in {time.time() - t0:.0f}s", flush=True)
    for i, bt in enumerate(batches(a.batches, seed=3)):
        db.append(measure_batch(torch, bt))
    print(f"collected {a.batches} batches in {time.time() - t0:.0f}s", flush=True)
    key = device_key(torch)
    (out / "tune_db.json").write_text(json.dumps(dict(device=key, rows=db)))
    w, hist = train(torch, db, steps=a.steps)
    write_weights(out / "picker_weights.bin", w, key)
    held = shapes(a.holdout, seed=2, hi=md)
    held_b = batches(a.holdout_batches, seed=4)
    summary, rows = evaluate(torch, pool, w, held, held_b, gen, key["sms"])
    report = dict(device=key, train=len(db), holdout=len(rows), max_dim=md, loss_history=hist, **summary,
                  seconds=round(time.time() - t0, 1))
    (out / "tune_report.json").write_text(json.dumps(dict(report, holdout_rows=rows)))
    print(json.dumps({k: v for k, v in report.items() if k != "loss_history"}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
