"""The N>1 host logic of bench.py on CPU (gloo, world size 2).

The timestep does not shard: N GPUs run N independent replicas and the job's
time is the slowest rank's.  These tests run that host logic as two gloo
ranks: the max-over-ranks reduction and throughput, and the reference arm
under torchrun, where rank 0 alone times the CPU reference and prints the one
JSON line while the other rank exits 0 without work.
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, results):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 10.0 + 5.0 * rank            # rank 1 is the slow replica
        got = bench.max_over_ranks(dist, ms, "cpu")
        results[rank] = (got, bench.replica_throughput(world, 1000.0, 4, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    port = _free_port()
    with mp.Manager() as m:
        results = m.dict()
        mp.start_processes(_rank_main, args=(2, port, results), nprocs=2, start_method="spawn", join=True)
        res = dict(results)
    assert res[0][0] == res[1][0] == 15.0
    # 2 replicas x 1000 cells x 4 steps in 15 ms
    assert res[0][1] == pytest.approx(2 * 1000 * 4 / 0.015)


def test_single_rank_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(None, 7.5, "cpu") == 7.5


def test_reference_arm_two_ranks_torchrun(oracle_lib):
    if not os.path.exists(oracle_lib.REF_BENCH_BIN):
        pytest.skip("reference benchmark binary not built")
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "2", "--warmup", "1", "--edge", "12"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT,
                       env=dict(os.environ, OMP_NUM_THREADS="2"))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2 and rec["steps"] == 2
    assert rec["value"] > 0 and rec["e2e"]["h2d_bytes_per_step"] == 0
    assert rec["cpu_baseline"]["kind"] == "reference"
