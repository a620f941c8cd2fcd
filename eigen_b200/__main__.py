"""Run and time products through the library from the command line.

    python -m eigen_b200 gemm --dtype d --method crt --m 4096 --n 4096 --k 4096 [--reps 3] [--r 0]
    python -m eigen_b200 batch --dtype d --count 10000 [--reps 3]
    python -m eigen_b200 level3 --routine trsm --chars LLNN --m 8192 --n 8192 [--k 8192] [--reps 3]

`gemm` runs C = A*B (NN, column-major, alpha = 1, beta = 0; --dtype z / c: the complex
product through zgemm_ / cgemm_, rated at 8mnk flops) on device-resident random
inputs (entries u*2^e, u ~ U[-1,1], e ~ U{-r..r}) with eb2_dgemm_device / eb2_sgemm_device
(method auto | native | emulated | crt; for SGEMM emulated means split-BF16), once to warm
up and then `reps` times, and prints one JSON line: the device time of each call (CUDA
events on the launching stream) and the library's record of the last call.  `batch` runs
the uneven 10,000-product batch of the benchmark as one grouped launch.  `level3` runs one of
the other level-3 routines (gemmtr, syrk, syr2k, symm, trmm, trsm; `--chars` its character
arguments in order) on device-resident operands through its BLAS symbol and reports the
routine's device time (CUDA events the library records on its stream) and its rate in the
routine's own flop count (syrk/gemmtr n(n+1)k, syr2k 2n(n+1)k, symm 2m^2n or 2mn^2, trmm/trsm
m^2n or mn^2).  Triangular operands of trsm get a dominant diagonal (entries of the stored
triangle ~ U[-1,1]/size, diagonal ~ +-U[1,2]).
"""
from __future__ import annotations

import argparse
import json
import sys

import eigen_b200 as eb

METHODS = {"auto": eb.METHOD_AUTO, "native": eb.METHOD_NATIVE, "emulated": eb.METHOD_EMULATED, "crt": eb.METHOD_CRT}


def time_complex_gemm(torch, dtype, m, n, k, reps, method="auto", seed=0) -> dict:
    """zgemm_ / cgemm_ (dtype "z" / "c") on device operands, NN, alpha = 1, beta = 0: the
    library's device time of each of `reps` calls after one warm-up, rated at 8mnk flops."""
    dt = torch.complex128 if dtype == "z" else torch.complex64
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    A = torch.randn((k, m), dtype=dt, device="cuda", generator=g)
    B = torch.randn((n, k), dtype=dt, device="cuda", generator=g)
    C = torch.zeros((n, m), dtype=dt, device="cuda")
    if dtype == "z":
        eb.set_dgemm_method(METHODS[method])
    else:
        eb.set_sgemm_method(METHODS[method] if method != "crt" else eb.METHOD_EMULATED)
    times = []
    for i in range(reps + 1):
        eb.complex_gemm(dtype, "N", "N", m, n, k, 1.0, A, m, B, k, 0.0, C, m)
        err = eb.last_error()
        if err[0] != eb.EB2_OK:
            return {"error": err}
        if i:
            times.append(eb.last_call_info()["kernel_ms"])
    best = min(times)
    return {"op": dtype + "gemm", "m": m, "n": n, "k": k, "method": method, "ms": [round(t, 4) for t in times],
            "tflops": round(8.0 * m * n * k / (best * 1e-3) / 1e12, 3), "call": eb.last_call_info()}


def _complex_gemm(a, torch):
    res = time_complex_gemm(torch, a.dtype, a.m, a.n, a.k, a.reps, a.method, a.seed)
    print(json.dumps(res))
    return 0 if "error" not in res else 1


def _gemm(a, torch):
    if a.dtype in ("z", "c"):
        return _complex_gemm(a, torch)
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


def time_level3(torch, routine, chars, dtype, m, n, k, reps, method="auto", seed=0) -> dict:
    """One of gemmtr, syrk, syr2k, symm, trmm, trsm (`chars` its character arguments in order)
    on device operands through its BLAS symbol: the library's device time of each of `reps`
    calls after one warm-up and the rate in the routine's own flop count."""
    dt = torch.float64 if dtype == "d" else torch.float32
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    ch = chars.upper()

    def rnd(rows, cols):
        return torch.rand((cols, rows), dtype=dt, device="cuda", generator=g) * 2 - 1  # column-major

    r = routine
    if r in ("gemmtr", "syrk", "syr2k"):
        ta = ch[1] != "N"
        tb = (ch[2] != "N") if r == "gemmtr" else not ta
        A = rnd(k, n) if ta else rnd(n, k)
        B = (rnd(n, k) if tb else rnd(k, n)) if r == "gemmtr" else (rnd(k, n) if ta else rnd(n, k))
        C = rnd(n, n)
        lda, ldb = A.shape[1], B.shape[1]
        args = {"gemmtr": [*ch, n, k, 1.0, A, lda, B, ldb, 0.5, C, n],
                "syrk": [*ch, n, k, 1.0, A, lda, 0.5, C, n],
                "syr2k": [*ch, n, k, 1.0, A, lda, B, ldb, 0.5, C, n]}[r]
        flops = (2 if r == "syr2k" else 1) * n * (n + 1) * k
        dims = {"n": n, "k": k}
    else:
        left = ch[0] == "L"
        size = m if left else n
        A = rnd(size, size)
        B = rnd(m, n)
        if r == "symm":
            C = rnd(m, n)
            args = [*ch, m, n, 1.0, A, size, B, m, 0.5, C, m]
            flops = 2 * size * m * n
        else:
            if r == "trsm":
                A = A / size
                d = (torch.rand(size, dtype=dt, device="cuda", generator=g) + 1) * torch.where(
                    torch.rand(size, device="cuda", generator=g) < 0.5, -1.0, 1.0).to(dt)
                A.diagonal().copy_(d)
            args = [*ch, m, n, 1.0, A, size, B, m]
            flops = size * m * n
        dims = {"m": m, "n": n}
    name = dtype + r
    if dtype == "d":
        eb.set_dgemm_method(METHODS[method])
    else:
        eb.set_sgemm_method(METHODS[method] if method != "crt" else eb.METHOD_EMULATED)
    out = B if r in ("trmm", "trsm") else C
    keep = out.clone()
    times = []
    for i in range(reps + 1):
        out.copy_(keep)  # trmm / trsm overwrite their operand: every call starts from the same B
        torch.cuda.synchronize()
        eb.level3(name, *args)
        err = eb.last_error()
        if err[0] != eb.EB2_OK:
            return {"error": err}
        if i:
            times.append(eb.last_call_info()["kernel_ms"])
    best = min(times)
    return {"op": name, "chars": chars, **dims, "method": method, "ms": [round(t, 4) for t in times],
            "tflops": round(flops / (best * 1e-3) / 1e12, 3), "call": eb.last_call_info()}


def _level3(a, torch):
    res = time_level3(torch, a.routine, a.chars, a.dtype, a.m, a.n, a.k, a.reps, a.method, a.seed)
    print(json.dumps(res))
    return 0 if "error" not in res else 1


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
    ap.add_argument("op", choices=["gemm", "batch", "level3"])
    ap.add_argument("--routine", choices=["gemmtr", "syrk", "syr2k", "symm", "trmm", "trsm"], default="trsm")
    ap.add_argument("--chars", default="LLNN", help="level3: the routine's character arguments, in order")
    ap.add_argument("--dtype", choices=["d", "s", "z", "c"], default="d",
                    help="z / c: complex GEMM through zgemm_ / cgemm_ (gemm only)")
    ap.add_argument("--method", choices=sorted(METHODS), default="auto")
    ap.add_argument("--m", type=int, default=4096)
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--k", type=int, default=4096)
    ap.add_argument("--r", type=int, default=0)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--count", type=int, default=10000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-check", action="store_true", help="DGEMM without the a-posteriori accuracy check")
    ap.add_argument("--tile", type=int, choices=[0, 128, 256, 512, 1024], default=0,
                    help="tcgen05 tile configuration (256: one CTA per 128x256 tile, 512: CTA pair, "
                         "1024: one CTA per 256x256 tile, CRT only; 0: per call)")
    a = ap.parse_args(argv)
    import torch

    eb.load()
    eb.set_timing(True)
    eb.set_tile_n(a.tile)
    return {"gemm": _gemm, "batch": _batch, "level3": _level3}[a.op](a, torch)


if __name__ == "__main__":
    sys.exit(main())
