"""The multi-rank plumbing of bench.py on CPU (gloo, world size 2).

bench.py runs one replica per GPU with no data-path collective; what crosses
ranks is the barrier around the timed region and the max over ranks of the
measured time.  These tests run that plumbing as two gloo ranks, and the
reference arm under torchrun, where rank 0 alone works and prints."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    bench.barrier(world)
    got = bench.max_over_ranks(float(10 * rank + 3), world, None)
    bench.barrier(world)
    dist.destroy_process_group()
    with open(os.path.join(out_dir, "rank%d.txt" % rank), "w") as f:
        f.write(repr(got))


def test_max_over_ranks_and_barrier_gloo(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    for r in range(world):
        assert float((tmp_path / ("rank%d.txt" % r)).read_text()) == 13.0


def test_max_over_ranks_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(1.25, 1) == 1.25
    bench.barrier(1)


def test_reference_arm_under_torchrun_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--nbody", "6", "--emax", "5", "--steps", "2", "--warmup", "1",
           "--ref-stride", "2"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300, env=env)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, p.stdout
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2
    assert rec["value"] > 0 and rec["e2e"]["h2d_bytes_per_step"] == 0
