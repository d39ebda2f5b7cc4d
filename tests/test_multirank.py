"""The multi-GPU form of the benchmark (replicas of the single-scene step) on CPU ranks over gloo:
the timing reduction is a max over ranks, the aggregate counts every replica's work, and the
reference arm runs on rank 0 only."""
import os
import socket
import subprocess
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    sys.path.insert(0, ROOT)
    import bench
    t = bench.max_over_ranks(0.5 + rank, dist, "cpu")
    out[rank] = (t, bench.aggregate_rate(world, 1000, 10, 5, t))
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_max_over_ranks_gloo(world):
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    slowest = 0.5 + (world - 1)
    for rank in range(world):
        t, rate = res[rank]
        assert t == slowest
        assert rate == pytest.approx(world * 1000 * 10 * 5 / slowest)


def test_reference_arm_only_on_rank0():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
