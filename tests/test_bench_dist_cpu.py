"""The bench's multi-process plumbing with two gloo ranks on the CPU: the
max-over-ranks timing and the reference arm under torch.distributed.run
(rank 0 measures and prints one JSON line; the other rank exits without
work).  The GPU arm's replicas use the same helpers with NCCL."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        v = bench.max_over_ranks(1.5 + rank, dist, "cpu")
        with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as f:
            f.write(repr(v))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    mp.start_processes(_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    vals = [float((tmp_path / f"r{r}.txt").read_text()) for r in (0, 1)]
    assert vals == [2.5, 2.5]


def test_max_over_ranks_single_process():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.25, None, "cpu") == 3.25


def test_reference_arm_under_torchrun_two_ranks():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py",
           "--impl", "reference", "--gpus", "2", "--nx", "64", "--ny", "32", "--steps", "1",
           "--warmup", "0"]
    env = dict(os.environ, OMP_NUM_THREADS="2", CUDA_VISIBLE_DEVICES="")
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["n_gpus"] == 2
    assert d["e2e"]["value"] == d["value"]
