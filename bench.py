#!/usr/bin/env python
"""FP64-accurate GEMM throughput on B200: the emulated DGEMM (Ozaki scheme II: INT8
residue products modulo 16 coprime moduli on tcgen05, exact CRT reconstruction) next to
the native FP64 DMMA kernel, at M = N = K = 8192.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--r R]

One step = one C = A*B product (NN, column-major, alpha = 1, beta = 0) of 8192^3 with
entries u*2^e, u ~ U[-1,1], e ~ U{-r..r} (r = 0 by default), through the library's
public entry points:
  * value: eb2_dgemm_device on device-resident inputs (automatic method, with the
    a-posteriori accuracy check), device time from CUDA events on the launching stream,
    max over ranks;
  * e2e:   dgemm_ (the Fortran BLAS ABI Eigen binds) on pinned host buffers: the H2D copy
    of A and B, the product and the D2H copy of C are inside the timed region;
  * roofline: the main tcgen05 GEMM kernel, timed by CUDA events recorded around it on
    its own stream; its DRAM traffic comes from the committed ncu summary;
  * cpu_baseline: Eigen's own multithreaded CPU GEMM (operator*, OpenMP) built from the
    reference sources (oracle/_ref), on a bounded sample, rank 0 only.
Multi-GPU: replicas only (every rank computes its own product; no collective on the data
path); the barrier and the MAX over ranks of the step time use NCCL.
`--impl reference` times the reference's CPU implementation on the same config.
"""
from __future__ import annotations

import argparse
import ctypes
import datetime
import json
import os
import re
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "FP64-accurate GEMM TFLOP/s (emulated vs native, 8192^3); grouped-batch GFLOP/s"
UNIT = "TFLOP/s"
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_BF16_TFLOPS = 1590.0
FALLBACK_HBM_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--size", type=int, default=8192)
    ap.add_argument("--r", type=int, default=0, help="exponent range of the synthetic entries")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-native", action="store_true")
    ap.add_argument("--no-grouped", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--no-sgemm", action="store_true", help="skip the split-BF16 / native FP32 SGEMM leg")
    ap.add_argument("--no-level3", action="store_true", help="skip the level-3 routine and complex GEMM leg")
    ap.add_argument("--no-sweep", action="store_true", help="skip the native-precision sweep (C2) leg")
    a = ap.parse_args()
    a.warmup = max(a.warmup, 3)
    a.steps = max(a.steps, 1)
    return a


def workload_config(a) -> dict:
    s = a.size
    return {
        "workload": f"emulated DGEMM {s}^3 NN column-major, alpha=1, beta=0, entries u*2^e (u~U[-1,1], e~U{{-{a.r}..{a.r}}})",
        "m": s, "n": s, "k": s, "dtype_inputs": "f64", "exponent_range_r": a.r,
        "l2": f"inputs larger than L2 ({s * s * 8 / 1e6:.0f} MB per operand vs 126 MB L2), no flush",
        "parallelism": f"replicas x{a.gpus}",
    }


# ------------------------------------------------------------------------ distributed
def dist_setup(a):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(dist, x: float, world: int, device) -> float:
    """The slowest rank's time (every rank takes part, in the same order)."""
    if world == 1:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_tflops(world: int, flops_per_rank: float, ms_max: float) -> float:
    """Replicas: every rank computes its own product; the job's throughput is all ranks'
    flops over the slowest rank's time."""
    return world * flops_per_rank / (ms_max * 1e-3) / 1e12


def host_cpu_info():
    model, flags = "unknown", ""
    try:
        txt = Path("/proc/cpuinfo").read_text()
        m = re.search(r"^model name\s*:\s*(.*)$", txt, re.M)
        model = m.group(1).strip() if m else model
        f = re.search(r"^flags\s*:\s*(.*)$", txt, re.M)
        flags = f.group(1) if f else ""
    except OSError:
        pass
    return model, flags


def ref_bench_binary():
    _, flags = host_cpu_info()
    v4 = ROOT / "oracle" / "_ref" / "eigen_ref_bench_v4"
    v3 = ROOT / "oracle" / "_ref" / "eigen_ref_bench_v3"
    if "avx512f" in flags.split() and v4.exists():
        return v4
    return v3 if v3.exists() else None


def run_ref_bench(args_list, timeout=600):
    exe = ref_bench_binary()
    if exe is None:
        return None, "oracle/_ref/eigen_ref_bench_* not built (make -C oracle ref)"
    env = dict(os.environ)
    threads = os.cpu_count() or 1
    env.setdefault("OMP_NUM_THREADS", str(threads))
    r = subprocess.run([str(exe), *args_list], capture_output=True, text=True, timeout=timeout, env=env)
    if r.returncode != 0:
        return None, f"eigen_ref_bench failed: {r.stderr.strip()[:200]}"
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1]
    return json.loads(line), None


def cpu_sample(a, reps, warmup):
    """Eigen operator* on the box's cores: the full M=N=size product with K cut so one
    repetition stays near a second; throughput (TFLOP/s) is what is compared."""
    probe, err = run_ref_bench(["--mode", "gemm", "--m", str(a.size), "--n", str(a.size), "--k", "256", "--reps", "1",
                                "--warmup", "1"])
    if probe is None:
        return None, err
    gflops = max(probe["gflops"], 1.0)
    k_for_1s = int(gflops * 1e9 / (2.0 * a.size * a.size))
    k = max(256, min(a.size, (k_for_1s // 256) * 256))
    res, err = run_ref_bench(["--mode", "gemm", "--m", str(a.size), "--n", str(a.size), "--k", str(k), "--reps",
                              str(reps), "--warmup", str(warmup), "--max-seconds", "25"])
    if res is None:
        return None, err
    res["k_sample"] = k
    return res, None


# ------------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_id: str | None):
        self.proc = None
        self.device_id = device_id

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "50"]
        if self.device_id:
            cmd += ["-i", self.device_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self) -> dict | None:
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        rows = [r.split(",") for r in out.strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        loaded = sorted(sm)[len(sm) // 2:] if sm else []
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------------ peaks / profiles
def level3_cpu_reference(n=2048, nz=1024):
    """The reference's own level-3 routines and complex GEMM (Eigen's BLAS library built from
    the reference sources into oracle/_ref, as its BLAS shim runs them: one thread per call) on a
    bounded sample: one call each after a small warm-up, n = 2048 (complex: 1024)."""
    import ctypes

    import numpy as np

    path = ROOT / "oracle" / "_ref" / "libeigen_ref_blas.so"
    if not path.exists():
        return {"error": "oracle/_ref/libeigen_ref_blas.so not built (make -C oracle ref)"}
    lib = ctypes.CDLL(str(path), mode=ctypes.RTLD_LOCAL)
    rng = np.random.default_rng(0)
    i, d = ctypes.c_int, ctypes.c_double
    P = lambda x: ctypes.c_void_p(x.ctypes.data)  # noqa: E731
    R = ctypes.byref

    def calls(m):
        A = np.asfortranarray(rng.uniform(-1, 1, (m, m)))
        B = np.asfortranarray(rng.uniform(-1, 1, (m, m)))
        C = np.asfortranarray(rng.uniform(-1, 1, (m, m)))
        T = np.asfortranarray(np.tril(A) / m + 1.5 * np.eye(m))
        Z = np.asfortranarray(A + 1j * B)
        W = np.asfortranarray(B + 1j * A)
        Y = np.zeros((m, m), complex, order="F")
        one, half = d(1.0), d(0.5)
        zal, zbe = (d * 2)(1.0, 0.0), (d * 2)(0.0, 0.0)
        M = i(m)
        return {
            "dsyrk UN": (lambda: lib.dsyrk_(b"U", b"N", R(M), R(M), R(one), P(A), R(M), R(half), P(C), R(M)),
                         m * (m + 1) * m),
            "dsymm LU": (lambda: lib.dsymm_(b"L", b"U", R(M), R(M), R(one), P(A), R(M), P(B), R(M), R(half), P(C),
                                            R(M)), 2 * m ** 3),
            "dtrmm LLNN": (lambda: lib.dtrmm_(b"L", b"L", b"N", b"N", R(M), R(M), R(one), P(T), R(M), P(B), R(M)),
                           m ** 3),
            "dtrsm LLNN": (lambda: lib.dtrsm_(b"L", b"L", b"N", b"N", R(M), R(M), R(one), P(T), R(M), P(B), R(M)),
                           m ** 3),
            "zgemm NN": (lambda: lib.zgemm_(b"N", b"N", R(M), R(M), R(M), zal, P(Z), R(M), P(W), R(M), zbe, P(Y),
                                            R(M)), 8 * m ** 3),
        }

    for f, _ in calls(128).values():  # warm-up: code and page faults
        f()
    out = {}
    for name, (f, flops) in calls(n).items():
        if name.startswith("zgemm"):
            f, flops = calls(nz)[name]
        t0 = time.perf_counter()
        f()
        dt = time.perf_counter() - t0
        out[name] = {"size": nz if name.startswith("zgemm") else n, "s": round(dt, 3),
                     "tflops": round(flops / dt / 1e12, 5)}
    return out


def peaks():
    try:
        p = json.loads(PEAKS_FILE.read_text())
        return float(p["bf16_tflops"]), float(p["bf16_tflops_sustained"]), float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_BF16_TFLOPS, 1400.0, FALLBACK_HBM_GBS, "fallback"


# The main GEMM kernel's instantiation for a method and tile configuration (tile 512 = CTA pair,
# 1024 = one CTA per 256x256 tile).
def gemm_instantiation(method_crt: bool, tile: int) -> str:
    if method_crt:
        return {512: "slice_gemm_kernel<2, 256, 6, 4, true>",
                1024: "slice_gemm_kernel<2, 256, 3, 16, false, 2>"}.get(tile, "slice_gemm_kernel<2, 256, 4, 4, false>")
    return "slice_gemm_kernel<0, 128, 8, 8, true>" if tile == 512 else "slice_gemm_kernel<0, 128, 6, 8, false>"


def profiled_traffic(size: int, instantiation: str):
    """DRAM bytes per launch of `instantiation` at `size`^3 from the committed ncu summaries
    (a line 'dram_bytes_per_launch: <bytes> at <size> for <instantiation>' in profiles/*.md),
    with the file it came from; (None, None) when no summary covers that kernel and size."""
    pat = re.compile(r"dram_bytes_per_launch:\s*([0-9.eE+]+)\s*at\s*(\d+)\s*for\s*(\S.*\S)\s*$", re.M)
    for f in sorted((ROOT / "profiles").glob("*.md")):
        for m in pat.finditer(f.read_text()):
            if int(m.group(2)) == size and m.group(3).strip("` ") == instantiation:
                return float(m.group(1)), f"profiles/{f.name}"
    return None, None


# ------------------------------------------------------------------------ end-to-end legs
def pageable_e2e_leg(eb, A, B, S, steps, rank_max, world):
    """dgemm_ on ordinary (pageable) numpy buffers, as a C or Fortran caller with malloc'd
    matrices calls it: beta = 0 (C not read) and beta = 1 (C copied in as well, what Eigen's
    operator* passes); host-timed synchronous calls, copies included."""
    import numpy as np

    hA = np.asfortranarray(A.cpu().numpy().T)  # column-major S x S, pageable
    hB = np.asfortranarray(B.cpu().numpy().T)
    hC = np.zeros((S, S), order="F")
    out = {}
    for beta in (0.0, 1.0):
        eb.dgemm("N", "N", S, S, S, 1.0, hA, S, hB, S, beta, hC, S)  # warm-up (staging buffers)
        times = []
        for _ in range(steps):
            t0 = time.perf_counter()
            eb.dgemm("N", "N", S, S, S, 1.0, hA, S, hB, S, beta, hC, S)
            times.append(time.perf_counter() - t0)
        t = rank_max(float(np.median(times)))
        out[f"beta{int(beta)}"] = {
            "value": round(whole_job_tflops(world, 2.0 * S ** 3, t * 1e3), 3), "unit": UNIT,
            "ms_per_step": round(t * 1e3, 3), "steps": steps,
            "h2d_bytes_per_step": (2 + int(beta != 0.0)) * S * S * 8, "d2h_bytes_per_step": S * S * 8}
    out["api"] = "dgemm_ (Fortran BLAS ABI) on pageable host buffers; synchronous call timed on the host"
    return out


def eigen_seam_leg(S, reps=3):
    """Eigen's operator* (C.noalias() = A * B on pageable MatrixXd) compiled with EIGEN_USE_BLAS
    against the reference headers and linked to the library (tests/eigen_seam/eigen_seam_bench):
    beta = 1 after Eigen's setZero, so C is copied in too; host-timed, median of `reps`."""
    exe = ROOT / "tests" / "eigen_seam" / "_bin" / "eigen_seam_bench"
    if not exe.exists():
        return {"error": "tests/eigen_seam/_bin/eigen_seam_bench not built (make -C tests/eigen_seam REF=...)"}
    r = subprocess.run([str(exe), str(S), str(reps), "1"], capture_output=True, text=True, timeout=900)
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    if r.returncode != 0 or not lines:
        return {"error": f"eigen_seam_bench rc={r.returncode}: {(r.stderr or r.stdout).strip()[:200]}"}
    res = json.loads(lines[-1])
    return {"value": round(res["tflops"], 3), "unit": UNIT, "ms_per_step": round(res["seconds_median"] * 1e3, 3),
            "steps": res["reps"], "h2d_bytes_per_step": 3 * S * S * 8, "d2h_bytes_per_step": S * S * 8,
            "method": res["method"], "moduli_or_slices": res["slices"], "spot_rel_err": res["spot_rel_err"],
            "api": "Eigen MatrixXd operator* (C.noalias() = A * B) through EIGEN_USE_BLAS -> dgemm_, pageable"}


# ------------------------------------------------------------------------ native sweep
def native_sweep_leg(eb, torch, dev, rank_max, sizes=(1024, 2048, 4096, 8192), reps=3):
    """The native-precision sweep: DGEMM and SGEMM at M = N = K in `sizes`, NN / NT / TN,
    alpha = 1.5, beta = 0.5, A, B, C ~ U[-1,1], leading dimensions + 8, through the device entry
    points with the native kernels (FP64 DMMA, FP32 FFMA) and with the default method (CRT
    emulation / split-BF16): TFLOP/s (2MNK over the CUDA-event time of one call, best of
    `reps` after a warm-up), max over ranks."""
    out = []
    stream = torch.cuda.Stream(device=dev)
    g = torch.Generator(device=dev)
    for dtype, tdt in (("d", torch.float64), ("s", torch.float32)):
        for S in sizes:
            ld = S + 8
            g.manual_seed(S)
            A = (torch.rand((S, ld), dtype=torch.float64, device=dev, generator=g) * 2 - 1).to(tdt)
            B = (torch.rand((S, ld), dtype=torch.float64, device=dev, generator=g) * 2 - 1).to(tdt)
            C0 = (torch.rand((S, ld), dtype=torch.float64, device=dev, generator=g) * 2 - 1).to(tdt)
            C = C0.clone()
            for ta, tb in (("N", "N"), ("N", "T"), ("T", "N")):
                row = {"dtype": dtype, "size": S, "trans": ta + tb}
                for name, method in (("native", eb.METHOD_NATIVE), ("default", eb.METHOD_AUTO)):
                    if dtype == "d":
                        eb.set_dgemm_method(method)
                        call = lambda: eb.dgemm_device(ta, tb, S, S, S, 1.5, A, ld, B, ld, 0.5, C, ld,  # noqa: E731
                                                       stream=stream.cuda_stream, check_accuracy=True)
                    else:
                        eb.set_sgemm_method(method)
                        call = lambda: eb.sgemm_device(ta, tb, S, S, S, 1.5, A, ld, B, ld, 0.5, C, ld,  # noqa: E731
                                                       stream=stream.cuda_stream)
                    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    best = None
                    for i in range(reps + 1):
                        C.copy_(C0)
                        torch.cuda.synchronize()
                        ev0.record(stream)
                        rc = call()
                        ev1.record(stream)
                        stream.synchronize()
                        assert rc == eb.EB2_OK, eb.last_error()
                        if i:
                            t = ev0.elapsed_time(ev1)
                            best = t if best is None else min(best, t)
                    ms = rank_max(best)
                    row[name] = {"tflops": round(2.0 * S ** 3 / (ms * 1e-3) / 1e12, 3), "ms": round(ms, 4),
                                 "method": eb.last_call_info()["method"]}
                out.append(row)
            del A, B, C0, C
    eb.set_dgemm_method(eb.METHOD_AUTO)
    eb.set_sgemm_method(eb.METHOD_AUTO)
    return out


# ------------------------------------------------------------------------ grouped batch
def batch_sizes(count, seed):
    """m, n, k each round(exp(U[ln 3, ln 256])); with probability 0.2 all three from {3,4,6,8}."""
    import numpy as np

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        if rng.random() < 0.2:
            s = int(rng.choice([3, 4, 6, 8]))
            out.append((s, s, s))
        else:
            out.append(tuple(int(round(float(np.exp(rng.uniform(np.log(3.0), np.log(256.0)))))) for _ in range(3)))
    return out


def grouped_bench(eb, torch, dev, stream, steps, warmup, count=10000, seed=7):
    """10,000 uneven products per dtype: one graph-captured grouped launch vs one plain
    launch of the native kernel per product (eb2_gemm_each); both device-timed."""
    sizes = batch_sizes(count, seed)
    res = {}
    for dtype, tdt in (("d", torch.float64), ("s", torch.float32)):
        na = sum(m * k for m, n, k in sizes)
        nb = sum(k * n for m, n, k in sizes)
        nc = sum(m * n for m, n, k in sizes)
        g = torch.Generator(device=dev)
        g.manual_seed(seed)
        bufA = torch.rand(na + 2 * count, dtype=tdt, device=dev, generator=g) * 2 - 1
        bufB = torch.rand(nb + 2 * count, dtype=tdt, device=dev, generator=g) * 2 - 1
        bufC = torch.zeros(nc + 2 * count, dtype=tdt, device=dev)
        es = bufA.element_size()
        oa = ob = oc = 0
        probs = []
        for (m, n, k) in sizes:
            probs.append(dict(m=m, n=n, k=k, alpha=1.0, beta=0.0, a=bufA.data_ptr() + oa * es, lda=m,
                              b=bufB.data_ptr() + ob * es, ldb=k, c=bufC.data_ptr() + oc * es, ldc=m))
            oa += m * k + (m * k) % 2
            ob += k * n + (k * n) % 2
            oc += m * n + (m * n) % 2
        arr = eb.problems_array(probs)
        flops = float(sum(2.0 * m * n * k for m, n, k in sizes))
        plan = eb.GroupedPlan(dtype, arr)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                plan.execute(stream.cuda_stream)
            stream.synchronize()
            ev0.record(stream)
            for _ in range(steps):
                plan.execute(stream.cuda_stream)
            ev1.record(stream)
            stream.synchronize()
            ms_grouped = ev0.elapsed_time(ev1) / steps
            eb.gemm_each(dtype, arr, stream.cuda_stream)  # warm-up of the per-call path
            stream.synchronize()
            reps = max(1, min(3, steps))
            ev0.record(stream)
            for _ in range(reps):
                eb.gemm_each(dtype, arr, stream.cuda_stream)
            ev1.record(stream)
            stream.synchronize()
            ms_each = ev0.elapsed_time(ev1) / reps
        plan.close()
        res["fp64" if dtype == "d" else "fp32"] = {
            "gflops": round(flops / (ms_grouped * 1e-3) / 1e9, 1), "ms": round(ms_grouped, 4),
            "per_call_ms": round(ms_each, 3), "per_call_gflops": round(flops / (ms_each * 1e-3) / 1e9, 2),
            "speedup_vs_per_call": round(ms_each / ms_grouped, 1), "problems": count, "flops": flops,
            "launches": 1, "per_call_launches": count,
        }
        del bufA, bufB, bufC
    return res


def grouped_cpu_reference(count=10000):
    """The reference's CPU path for the same batch law (oracle/_ref/eigen_ref_bench --mode batch):
    an OpenMP parallel for over the products on all host threads, each C = A * B through Eigen's
    operator*, with fixed-size Matrix<Scalar,N,N> types (unrolled coefficient-based products)
    for the products drawn from {3,4,6,8}; median of 3 repetitions after a warm-up."""
    out = {}
    for dtype, key in (("d", "fp64"), ("s", "fp32")):
        res, err = run_ref_bench(["--mode", "batch", "--dtype", dtype, "--count", str(count), "--reps", "3",
                                  "--warmup", "1", "--max-seconds", "20"])
        if res is None:
            out[key] = {"error": err}
            continue
        out[key] = {"gflops": round(res["gflops"], 2), "ms": round(res["seconds_median"] * 1e3, 3),
                    "threads": res["threads"], "problems": res["count"],
                    "sample": "same size law (m, n, k log-uniform in [3, 256], 20% from {3,4,6,8} cubes), "
                              "its own seeded draw; Eigen operator* per product, OpenMP over products"}
    return out


# ------------------------------------------------------------------------ accuracy
def _exact_block(Ar, Bc):
    """alpha*A*B on a sampled block, rounded once from the exact sum: every product a*b is
    split exactly into hi + lo (Dekker), and math.fsum adds them without intermediate error."""
    import math

    import numpy as np

    split = 134217729.0  # 2^27 + 1

    def halves(x):
        t = x * split
        hi = t - (t - x)
        return hi, x - hi

    out = np.empty((Ar.shape[0], Bc.shape[1]))
    for i in range(Ar.shape[0]):
        a = Ar[i][:, None]
        p = a * Bc
        ah, al = halves(np.broadcast_to(a, Bc.shape))
        bh, bl = halves(Bc)
        e = ((ah * bh - p) + ah * bl + al * bh) + al * bl  # exact error of each product
        for j in range(Bc.shape[1]):
            out[i, j] = math.fsum(np.concatenate([p[:, j], e[:, j]]))
    return out


def sgemm_leg(eb, torch, dev, S, steps, rank_max, seed=123, sample=24):
    """Split-BF16 SGEMM (the default FP32 method) and the native FP32 kernel at S^3 on device
    operands: CUDA-event time over `steps` calls (max over ranks), and the normwise error of a
    sampled block against the FP64 product of the same FP32 inputs."""
    import numpy as np

    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    A = torch.rand((S, S), dtype=torch.float32, device=dev, generator=g) * 2 - 1
    B = torch.rand((S, S), dtype=torch.float32, device=dev, generator=g) * 2 - 1
    rng = np.random.default_rng(seed)
    rows = np.sort(rng.choice(S, sample, replace=False))
    cols = np.sort(rng.choice(S, sample, replace=False))
    # column-major: A(i, l) is A_t[l, i]; the FP64 product of FP32 inputs is exact to ~1e-16
    ref = A[:, rows].T.cpu().double().numpy() @ B[cols, :].T.cpu().double().numpy()
    out = {}
    stream = torch.cuda.Stream(device=dev)
    for name, method, n in (("split_bf16", eb.METHOD_EMULATED, steps), ("native_fp32", eb.METHOD_NATIVE, min(steps, 3))):
        eb.set_sgemm_method(method)
        C = torch.zeros((S, S), dtype=torch.float32, device=dev)
        for _ in range(2):
            assert eb.sgemm_device("N", "N", S, S, S, 1.0, A, S, B, S, 0.0, C, S, stream=stream.cuda_stream) == eb.EB2_OK
        stream.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(n):
            rc = eb.sgemm_device("N", "N", S, S, S, 1.0, A, S, B, S, 0.0, C, S, stream=stream.cuda_stream)
            assert rc == eb.EB2_OK, eb.last_error()
        ev1.record(stream)
        stream.synchronize()
        info = eb.last_call_info()
        ms = rank_max(ev0.elapsed_time(ev1) / n)
        got = C[cols][:, rows].T.cpu().double().numpy()
        out[name] = {"tflops": round(2.0 * S**3 / ms / 1e9, 3), "ms_per_step": round(ms, 3), "steps": n,
                     "rel_error": float(np.linalg.norm(got - ref) / np.linalg.norm(ref)),
                     "method": info["method"], "bf16_products": info["slices"]}
    eb.set_sgemm_method(eb.METHOD_AUTO)
    out["sample"] = f"{sample}x{sample} block of C against the FP64 product of the FP32 inputs"
    del A, B, C
    return out


def accuracy_leg(eb, torch, dev, S, r_values, seed=99, sample=24):
    """Normwise error of the automatic (emulated) and the native DGEMM against an exactly
    rounded reference on a sampled sub-block, for entries u*2^e with e in [-r, r]:
    ||dC||_F / ||C||_F, ||dC||_F / || |A||B| ||_F and max |dC| on the block."""
    import numpy as np

    out = {}
    g = torch.Generator(device=dev)
    rng = np.random.default_rng(seed)
    for r in r_values:
        g.manual_seed(seed + r)
        A = torch.rand((S, S), dtype=torch.float64, device=dev, generator=g) * 2 - 1
        B = torch.rand((S, S), dtype=torch.float64, device=dev, generator=g) * 2 - 1
        if r:
            A = torch.ldexp(A, torch.randint(-r, r + 1, (S, S), device=dev, generator=g).to(torch.float64))
            B = torch.ldexp(B, torch.randint(-r, r + 1, (S, S), device=dev, generator=g).to(torch.float64))
        rows = np.sort(rng.choice(S, sample, replace=False))
        cols = np.sort(rng.choice(S, sample, replace=False))
        # column-major: A(i, l) is A_t[l, i]
        Ar = A[:, rows].T.cpu().numpy().astype(np.float64)
        Bc = B[cols, :].T.cpu().numpy().astype(np.float64)
        ref = _exact_block(Ar, Bc)
        absprod = np.abs(Ar) @ np.abs(Bc)  # |A||B| on the block (rounding here is immaterial)
        res = {}
        for name, method in (("emulated", eb.METHOD_AUTO), ("native", eb.METHOD_NATIVE)):
            eb.set_dgemm_method(method)
            C = torch.zeros((S, S), dtype=torch.float64, device=dev)
            rc = eb.dgemm_device("N", "N", S, S, S, 1.0, A, S, B, S, 0.0, C, S, check_accuracy=True)
            torch.cuda.synchronize()
            info = eb.last_call_info()
            got = C[cols][:, rows].T.cpu().numpy()
            err = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
            res[name] = {"rel_error": err,
                         "rel_to_abs_product": float(np.linalg.norm(got - ref) / np.linalg.norm(absprod)),
                         "max_abs_error": float(np.max(np.abs(got - ref))),
                         "rc": rc, "method": info["method"], "moduli_or_slices": info["slices"],
                         "escalations": info["escalations"], "err_estimate": info["err_estimate"]}
        eb.set_dgemm_method(eb.METHOD_AUTO)
        res["sample"] = f"{sample}x{sample} block of C, exactly rounded reference"
        out[f"r{r}"] = res
        del A, B, C
    return out


# ------------------------------------------------------------------------ arms
def reference_arm(a, world, rank):
    cfg = workload_config(a)
    if rank != 0:
        return 0
    model, _ = host_cpu_info()
    res, err = run_ref_bench(["--mode", "gemm", "--m", str(a.size), "--n", str(a.size), "--k", "256", "--reps", "1"])
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return 0
    gflops = max(res["gflops"], 1.0)
    k = max(256, min(a.size, (int(gflops * 1e9 / (2.0 * a.size * a.size)) // 256) * 256))
    res, err = run_ref_bench(["--mode", "gemm", "--m", str(a.size), "--n", str(a.size), "--k", str(k), "--reps",
                              str(a.steps), "--warmup", str(a.warmup), "--max-seconds", "150"])
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return 0
    tflops = res["gflops"] / 1e3
    sample = (f"Eigen operator* (OpenMP, {res['threads']} threads, {model}) on {a.size}x{a.size}x{k} per step "
              f"(K cut from {a.size} to bound the step), {res['reps']} steps, median")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(tflops, 4), "unit": UNIT, "n_gpus": a.gpus,
        "steps": res["reps"], "warmup": a.warmup, "ms_per_step": round(res["seconds_median"] * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": cfg,
        "cpu_baseline": {"value": round(tflops, 4), "unit": UNIT, "cores": res["threads"], "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(tflops, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# The other level-3 routines and the complex GEMM, on device operands at the benchmark size,
# through their BLAS symbols with the default method: (routine, character arguments, dtype).
LEVEL3_CASES = [("syrk", "UN", "d"), ("gemmtr", "UNT", "d"), ("symm", "LU", "d"), ("trmm", "LLNN", "d"),
                ("trsm", "LLNN", "d"), ("trsm", "LLNN", "s"), ("zgemm", "NN", "z"), ("cgemm", "NN", "c")]


def level3_leg(torch, S, reps=3):
    """Device time (the library's events around each call, best of `reps` after a warm-up) and
    rate in each routine's own flop count; see eigen_b200.__main__."""
    from eigen_b200.__main__ import time_complex_gemm, time_level3

    out = []
    for routine, chars, dtype in LEVEL3_CASES:
        if dtype in ("z", "c"):
            res = time_complex_gemm(torch, dtype, S, S, S, reps)
        else:
            res = time_level3(torch, routine, chars, dtype, S, S, S, reps)
        if "error" in res:
            out.append({"op": dtype + routine, "error": res["error"]})
            continue
        call = res["call"]
        out.append({"op": res["op"], "chars": chars, "size": S, "ms": min(res["ms"]), "tflops": res["tflops"],
                    "method": call["method"], "moduli_or_slices": call["slices"],
                    "err_estimate": call["err_estimate"], "launches": call["launches"]})
    return out


def our_arm(a, world, rank, local):
    import torch
    import torch.distributed as dist

    import eigen_b200 as eb

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    props = torch.cuda.get_device_properties(dev)
    pci = None
    if hasattr(props, "pci_bus_id"):
        pci = f"{getattr(props, 'pci_domain_id', 0):08X}:{props.pci_bus_id:02X}:{getattr(props, 'pci_device_id', 0):02X}.0"
    eb.load()
    S = a.size
    flops = 2.0 * S ** 3
    g = torch.Generator(device=dev)
    g.manual_seed(1234 + rank)

    def synth(rows, cols):
        # column-major rows x cols == row-major (cols, rows) tensor
        x = torch.rand((cols, rows), dtype=torch.float64, device=dev, generator=g) * 2 - 1
        if a.r:
            e = torch.randint(-a.r, a.r + 1, (cols, rows), device=dev, generator=g, dtype=torch.int32)
            x = torch.ldexp(x, e.to(torch.float64))
        return x

    A = synth(S, S)
    B = synth(S, S)
    C = torch.zeros((S, S), dtype=torch.float64, device=dev)
    stream = torch.cuda.Stream(device=dev)
    eb.set_dgemm_method(eb.METHOD_AUTO)
    eb.set_timing(True)

    def barrier():
        if world > 1:
            dist.barrier()

    def rank_max(x: float) -> float:
        return max_over_ranks(dist, x, world, dev)

    def run_device(method, steps):
        eb.set_dgemm_method(method)
        infos = []
        with torch.cuda.stream(stream):
            for _ in range(a.warmup):
                rc = eb.dgemm_device("N", "N", S, S, S, 1.0, A, S, B, S, 0.0, C, S, stream=stream.cuda_stream,
                                     check_accuracy=True)
                assert rc == eb.EB2_OK, eb.last_error()
            stream.synchronize()
            barrier()
            torch.cuda.synchronize()
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            for _ in range(steps):
                rc = eb.dgemm_device("N", "N", S, S, S, 1.0, A, S, B, S, 0.0, C, S, stream=stream.cuda_stream,
                                     check_accuracy=True)
                assert rc == eb.EB2_OK, eb.last_error()
                infos.append(eb.last_call_info())
            ev1.record(stream)
            stream.synchronize()
        barrier()
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / steps
        return ms, infos

    clocks = ClockSampler(pci)
    clocks.start()
    time.sleep(0.3)
    ms_emu, infos = run_device(eb.METHOD_AUTO, a.steps)
    clk = clocks.stop()
    ms_emu_max = rank_max(ms_emu)
    C_emu = C.clone()
    gemm_ms = [i["gemm_kernel_ms"] for i in infos if i["gemm_kernel_ms"] > 0]
    gemm_ms_avg = rank_max(sum(gemm_ms) / len(gemm_ms)) if gemm_ms else None
    slices = infos[-1]["slices"]
    launches = sum(i["launches"] for i in infos)
    # device time of one call's kernels (events around them inside the library), against which
    # ms_per_step also holds the host side of each synchronous, checked call
    call_ms = sorted(i["kernel_ms"] for i in infos if i["kernel_ms"] > 0)
    kernel_ms_per_call = round(call_ms[len(call_ms) // 2], 3) if call_ms else None

    native = None
    if not a.no_native:
        nsteps = min(a.steps, 5)
        ms_nat, _ = run_device(eb.METHOD_NATIVE, nsteps)
        ms_nat = rank_max(ms_nat)
        diff = float(torch.linalg.norm(C_emu - C) / torch.linalg.norm(C))
        native = {"tflops": round(whole_job_tflops(world, flops, ms_nat), 3), "ms_per_step": round(ms_nat, 3),
                  "steps": nsteps, "kernel": "dgemm_dmma (mma.sync f64)", "rel_diff_emulated_vs_native": diff}
        eb.set_dgemm_method(eb.METHOD_AUTO)

    e2e = None
    if not a.no_e2e:
        hA = torch.empty((S, S), dtype=torch.float64, pin_memory=True)
        hB = torch.empty((S, S), dtype=torch.float64, pin_memory=True)
        hC = torch.empty((S, S), dtype=torch.float64, pin_memory=True)
        hA.copy_(A)
        hB.copy_(B)
        e2e_steps = min(a.steps, 5)
        for _ in range(1):
            eb.dgemm("N", "N", S, S, S, 1.0, hA, S, hB, S, 0.0, hC, S)
        barrier()
        times = []
        for _ in range(e2e_steps):
            t0 = time.perf_counter()
            eb.dgemm("N", "N", S, S, S, 1.0, hA, S, hB, S, 0.0, hC, S)
            times.append(time.perf_counter() - t0)
        barrier()
        t_step = rank_max(sum(times) / len(times))
        e2e = {"value": round(whole_job_tflops(world, flops, t_step * 1e3), 3), "unit": UNIT,
               "h2d_bytes_per_step": 2 * S * S * 8, "d2h_bytes_per_step": S * S * 8,
               "ms_per_step": round(t_step * 1e3, 3), "steps": e2e_steps,
               "api": "dgemm_ (Fortran BLAS ABI) on pinned host buffers; synchronous call timed on the host"}

    e2e_pageable = e2e_eigen = None
    if not a.no_e2e:
        e2e_pageable = pageable_e2e_leg(eb, A, B, S, min(a.steps, 3), rank_max, world)
        if rank == 0 and world == 1:
            e2e_eigen = eigen_seam_leg(S, reps=3)

    accuracy = None
    if not a.no_accuracy:
        accuracy = accuracy_leg(eb, torch, dev, S, (0, 8, 32))

    sgemm = None
    if not a.no_sgemm:
        sgemm = sgemm_leg(eb, torch, dev, S, min(a.steps, 5), rank_max)

    grouped = None
    if not a.no_grouped:
        grouped = grouped_bench(eb, torch, dev, stream, a.steps, a.warmup)
        if rank == 0 and world == 1 and not a.no_cpu_baseline:
            grouped["cpu"] = grouped_cpu_reference()

    level3 = None
    if not a.no_level3:
        level3 = level3_leg(torch, S)

    sweep = None
    if not a.no_sweep:
        sweep = native_sweep_leg(eb, torch, dev, rank_max)

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        model, _ = host_cpu_info()
        res, err = cpu_sample(a, reps=3, warmup=1)
        if res is not None:
            cpu = {"value": round(res["gflops"] / 1e3, 4), "unit": UNIT, "cores": res["threads"], "kind": "reference",
                   "sample": f"Eigen operator* (OpenMP, {model}) on {S}x{S}x{res['k_sample']} DGEMM, "
                             f"{res['reps']} reps median after 1 warm-up"}
        else:
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": err}
        if not a.no_level3:
            cpu["level3_reference"] = level3_cpu_reference()

    bf16, bf16_sus, hbm, basis = peaks()
    method = infos[-1]["method"]
    tile = infos[-1]["tile_n"]
    # INT8 products of 2*M*N*K each: one per modulus (CRT) or one per digit pair (slices)
    products = slices if method == eb.METHOD_CRT else slices * (slices + 1) // 2
    roof = None
    if gemm_ms_avg and method != eb.METHOD_NATIVE:
        achieved = flops / (gemm_ms_avg * 1e-3) / 1e12  # FP64-equivalent TFLOP/s of the GEMM kernel
        # dense int8 rate = 2 x dense bf16 on sm_100.  The burst figure applies to a timed loop
        # shorter than 2 s (the power cap has not settled the clocks yet), the sustained one above
        timed_s = ms_emu_max * a.steps * 1e-3
        sustained = timed_s >= 2.0
        int8_peak = 2.0 * (bf16_sus if sustained else bf16)
        peak = int8_peak / products  # the FP64-equivalent ceiling of an int8 kernel doing `products` GEMMs
        shape = {512: "CTA pair, 256x256 tiles, cta_group::2",
                 1024: "one CTA, 256x256 tiles (two M=128 MMAs per K step)"}.get(tile, "one CTA, 128x256 tiles")
        inst = gemm_instantiation(method == eb.METHOD_CRT, tile)
        traffic, traffic_src = profiled_traffic(S, inst)
        roof = {"bound": "tensor", "achieved": round(achieved, 3), "peak": round(peak, 3), "unit": UNIT,
                "frac": round(achieved / peak, 4), "traffic": traffic,
                "kernel": f"{inst} (tcgen05.mma kind::i8, {shape}), {gemm_ms_avg:.3f} ms/launch",
                "traffic_source": traffic_src,
                "pipe": {"achieved_tops": round(achieved * products, 1), "peak_tops": round(int8_peak, 1),
                         "basis": f"peak = 2 x {basis} {'sustained' if sustained else 'burst'} dense bf16 "
                                  f"({bf16_sus if sustained else bf16} TFLOP/s), of {basis}; timed region "
                                  f"{timed_s:.2f} s ({'>=' if sustained else '<'} 2 s); {products} int8 products "
                                  f"of 2*M*N*K each",
                         "sustained_frac": round(achieved * products / (2.0 * bf16_sus), 4),
                         "burst_frac": round(achieved * products / (2.0 * bf16), 4)}}

    value = whole_job_tflops(world, flops, ms_emu_max)
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(ms_emu_max, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int8 residues (s32 accumulate) -> f64", "data": "synthetic",
            "config": dict(workload_config(a), method=method, moduli_or_slices=slices, tile_n=infos[-1]["tile_n"],
                           err_estimate=infos[-1]["err_estimate"], escalations=infos[-1]["escalations"],
                           kernel_ms_per_call=kernel_ms_per_call),
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": clk, "native_fp64": native, "accuracy": accuracy, "sgemm": sgemm, "grouped_batch": grouped,
            "level3_routines": level3, "native_sweep": sweep, "e2e_pageable": e2e_pageable,
            "e2e_eigen_operator": e2e_eigen,
            "emulated_over_native": round(value / native["tflops"], 3) if native else None,
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    a = parse_args()
    world, rank, local = dist_setup(a)
    if a.impl == "reference":
        return reference_arm(a, world, rank)
    return our_arm(a, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
