"""The trained picker re-timed live (GPU): on about 20 held-out problems of the committed tuning
report, the automatic call (the installed weights choose the configuration class and, for
DGEMM, the modulus count) is timed next to every configuration class of its kind forced in
turn.  The picker's total time must stay close to the best forced class per problem, and well
below the worst.
"""
from __future__ import annotations

import json

import numpy as np
import pytest

import eigen_b200 as eb

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

DATA = eb.LIB_PATH.parent.parent / "data"


@pytest.fixture(autouse=True)
def _defaults():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    eb.load()
    yield
    eb.set_config(-1)
    eb.set_dgemm_method(eb.METHOD_AUTO)
    eb.set_sgemm_method(eb.METHOD_AUTO)
    eb.set_dgemm_moduli(0)
    eb.set_dgemm_tolerance(2.0 ** -53)


def _time(fn, reps=5):
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        ev0.record()
        fn()
        ev1.record()
        torch.cuda.synchronize()
        ts.append(ev0.elapsed_time(ev1))
    return float(np.median(ts))


def test_picker_choice_against_live_best():
    raw = (DATA / "picker_weights.bin").read_bytes()
    count = int.from_bytes(raw[8:12], "little")
    w = np.frombuffer(raw[16:16 + 4 * count], dtype="<f4").astype(np.float32)
    assert eb.set_picker(w) == eb.EB2_OK
    rows = json.loads((DATA / "tune_report.json").read_text())["holdout_rows"]
    # problems of 0.05 .. 5 ms (live timing noise stays small against them), DGEMM and SGEMM
    cand = [r for r in rows if r["kind"] in ("d", "s") and 0.05 <= r["times_ms"][str(r["best"])] <= 5.0]
    rng = np.random.default_rng(0)
    pick = rng.choice(len(cand), size=min(20, len(cand)), replace=False)
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    t_auto = t_best = t_worst = 0.0
    for i in pick:
        r = cand[int(i)]
        m, n, k = r["m"], r["n"], r["k"]
        dt = torch.float64 if r["kind"] == "d" else torch.float32
        A = torch.rand((k, m), dtype=dt, device="cuda", generator=g) * 2 - 1
        B = torch.rand((n, k), dtype=dt, device="cuda", generator=g) * 2 - 1
        C = torch.zeros((n, m), dtype=dt, device="cuda")
        if r["kind"] == "d":
            eb.set_dgemm_tolerance(2.0 ** -53)
            call = lambda: eb.dgemm_device("N", "N", m, n, k, 1.0, A, m, B, k, 0.0, C, m, check_accuracy=True)
            classes = range(0, 6)
        else:
            call = lambda: eb.sgemm_device("N", "N", m, n, k, 1.0, A, m, B, k, 0.0, C, m)
            classes = range(6, 10)
        eb.set_config(-1)
        eb.set_dgemm_moduli(0)
        auto = _time(call)
        assert eb.last_error()[0] == eb.EB2_OK, eb.last_error()
        # the forced classes run the modulus count the automatic call settled on
        info = eb.last_call_info()
        eb.set_dgemm_moduli(info["slices"] if r["kind"] == "d" and info["method"] == eb.METHOD_CRT else 0)
        forced = []
        for c in classes:
            eb.set_config(c)
            forced.append(_time(call))
        eb.set_config(-1)
        t_auto += auto
        t_best += min(forced)
        t_worst += max(forced)
        del A, B, C
    assert t_auto <= 1.15 * t_best + 0.02 * len(pick), (t_auto, t_best, t_worst)
    assert t_auto < t_worst, (t_auto, t_best, t_worst)
