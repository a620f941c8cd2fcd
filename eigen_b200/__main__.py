"""Run and time products through the library from the command line.

    python -m eigen_b200 gemm --dtype d --method crt --m 4096 --n 4096 --k 4096 [--reps 3] [--r 0]
    python -m eigen_b200 batch --dtype d --count 10000 [--reps 3]

`gemm` runs C = A*B (NN, column-major, alpha = 1, beta = 0) on device-resident random
inputs (entries u*2^e, u ~ U[-1,1], e ~ U{-r..r}) with eb2_dgemm_device / eb2_sgemm_device
(method auto | native | emulated | crt; for SGEMM emulated means split-BF16), once to warm
up and then `reps` times, and prints one JSON line: the device time of each call (CUDA
events on the launching stream) and the library's record of the last call.  `batch` runs
the uneven 10,000-product batch of the benchmark as one grouped launch.
"""
from __future__ import annotations

import argparse
import json
import sys

import eigen_b200 as eb

METHODS = {"auto": eb.METHOD_AUTO, "native": eb.METHOD_NATIVE, "emulated": eb.METHOD_EMULATED, "crt": eb.METHOD_CRT}


def _gemm(a, torch):
    dt = torch.float64 if a.dtype == "d" else torch.float32
    g = torch.Generator(device="cuda")
    g.manual_seed(a.seed)

    def rnd(rows, cols):
        x = torch.rand((cols, rows), dtype=dt, device="cuda", generator=g) * 2 - 1  # column-major rows x cols
        if a.r:
            e = torch.randint(-a.r, a.r + 1, x.shape, device="cuda", generator=g).to(dt)
            x = x * torch.exp2(e)
        return x

    A, B = rnd(a.m, a.k), rnd(a.k, a.n)
    C = torch.zeros((a.n, a.m), dtype=dt, device="cuda")
    if a.dtype == "d":
        eb.set_dgemm_method(METHODS[a.method])
        call = lambda: eb.dgemm_device("N", "N", a.m, a.n, a.k, 1.0, A, a.m, B, a.k, 0.0, C, a.m,
                                       check_accuracy=not a.no_check)
    else:
        eb.set_sgemm_method(METHODS[a.method] if a.method != "crt" else eb.METHOD_EMULATED)
        call = lambda: eb.sgemm_device("N", "N", a.m, a.n, a.k, 1.0, A, a.m, B, a.k, 0.0, C, a.m)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    times = []
    for i in range(a.reps + 1):
        ev0.record()
        rc = call()
        ev1.record()
        torch.cuda.synchronize()
        if rc != eb.EB2_OK:
            print(json.dumps({"error": eb.last_error()}))
            return 1
        if i:
            times.append(ev0.elapsed_time(ev1))
    best = min(times)
    print(json.dumps({"op": "gemm", "dtype": a.dtype, "m": a.m, "n": a.n, "k": a.k, "method": a.method,
                      "ms": [round(t, 4) for t in times],
                      "tflops": round(2.0 * a.m * a.n * a.k / (best * 1e-3) / 1e12, 3),
                      "call": eb.last_call_info()}))
    return 0


def _batch(a, torch):
    import importlib.util
    from pathlib import Path

    spec = importlib.util.spec_from_file_location("eb2_bench", Path(__file__).resolve().parents[1] / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    res = bench.grouped_bench(eb, torch, torch.device("cuda"), torch.cuda.Stream(), a.reps, 1, count=a.count)
    print(json.dumps({"op": "batch", **res}))
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m eigen_b200", description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("op", choices=["gemm", "batch"])
    ap.add_argument("--dtype", choices=["d", "s"], default="d")
    ap.add_argument("--method", choices=sorted(METHODS), default="auto")
    ap.add_argument("--m", type=int, default=4096)
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--k", type=int, default=4096)
    ap.add_argument("--r", type=int, default=0)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--count", type=int, default=10000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-check", action="store_true", help="DGEMM without the a-posteriori accuracy check")
    a = ap.parse_args(argv)
    import torch

    eb.load()
    eb.set_timing(True)
    return _gemm(a, torch) if a.op == "gemm" else _batch(a, torch)


if __name__ == "__main__":
    sys.exit(main())
