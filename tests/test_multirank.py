"""Multi-rank plumbing of bench.py on CPU (gloo, world size 2): the max over ranks and the
reference arm's rank-0-only behaviour.  The GPU runs use the same code with NCCL."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        got = bench.max_over_ranks(10.0 + 5.0 * rank, world, dist, device="cpu")
        out[rank] = got
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    port = _free_port()
    out = mp.get_context("spawn").Manager().dict()   # no fork of a process that holds threads
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    assert out[0] == 15.0 and out[1] == 15.0


def test_max_over_ranks_single():
    import bench

    assert bench.max_over_ranks(3.5, 1, None) == 3.5


def _run_ref(rank: int) -> subprocess.CompletedProcess:
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1")
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2",
                           "--workload", "uniform16", "--n", "2000", "--steps", "1", "--warmup", "1",
                           "--ref-rows", "4"], env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_rank_zero_only():
    r1 = _run_ref(1)
    assert r1.returncode == 0, r1.stderr
    assert r1.stdout.strip() == ""
    r0 = _run_ref(0)
    assert r0.returncode == 0, r0.stderr
    line = json.loads(r0.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0
