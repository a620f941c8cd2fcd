"""bench.py's multi-rank plumbing on the CPU (no GPU): two gloo ranks on 127.0.0.1.

The product has no exchange step, so N GPUs run N replicas; the only collectives are the
barrier and the max over ranks of each timed quantity, and the job's throughput is all
ranks' work over the slowest rank's time.  The reference arm under torchrun runs on rank 0
alone and prints one line; the other ranks exit 0 without work.
"""
from __future__ import annotations

import importlib.util
import json
import os
import socket
import subprocess
import sys

import pytest

from _helpers import ORACLE_DIR, ROOT

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _bench():
    spec = importlib.util.spec_from_file_location("eb2_bench", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench = _bench()
        local_ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        ms_max = bench.max_over_ranks(dist, local_ms, world, "cpu")
        dist.barrier()
        out[rank] = (ms_max, bench.whole_job_tflops(world, 2.0 * 8192 ** 3, ms_max))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_throughput_gloo():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
        res = dict(out)
    assert res[0] == res[1]
    ms_max, tflops = res[0]
    assert ms_max == 15.0
    assert abs(tflops - 2 * 2.0 * 8192 ** 3 / 15e-3 / 1e12) < 1e-9


def test_single_rank_needs_no_collective():
    bench = _bench()
    assert bench.max_over_ranks(None, 3.5, 1, "cpu") == 3.5
    assert abs(bench.whole_job_tflops(1, 1e12, 1000.0) - 1.0) < 1e-12


@pytest.mark.skipif(not (ORACLE_DIR / "_ref" / "eigen_ref_bench_v3").exists(), reason="oracle/_ref not built")
def test_reference_arm_under_torchrun_prints_once():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), str(ROOT / "bench.py"), "--impl", "reference", "--gpus",
           "2", "--steps", "1", "--warmup", "3", "--size", "1024"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, env=env, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(ln) for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "reference"
