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


# ---- the sharded forms on CPU ranks: batched scenes split by body count, calibration scenes split
# in contiguous ranges with one all-reduce of the material gradients ----

@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_split_scenes_covers_and_balances(world):
    sys.path.insert(0, ROOT)
    import bench
    import numpy as np
    rng = np.random.default_rng(world)
    sizes = [int(v) for v in rng.integers(256, 8193, 97)]
    parts = bench.split_scenes(sizes, world)
    assert len(parts) == world
    flat = sorted(s for p in parts for s in p)
    assert flat == list(range(len(sizes)))  # every scene on exactly one rank
    loads = [sum(sizes[s] for s in p) for p in parts]
    # largest-first greedy: the spread of the loads is at most one scene
    assert max(loads) - min(loads) <= max(sizes)
    assert bench.split_scenes(sizes, world) == parts  # deterministic: every rank computes the same split


def test_rank_range_partitions():
    sys.path.insert(0, ROOT)
    import bench
    for n in (1, 7, 64):
        for world in (1, 2, 3, 8):
            got = [bench.rank_range(n, r, world) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == n
            assert all(got[k][1] == got[k + 1][0] for k in range(world - 1))


def _calib_worker(rank, world, port, out):
    """One rank of the calibration split: its scenes' loss gradient along (E, e, mu) by the
    oracle's dual numbers, summed over ranks by the all-reduce the benchmark does."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import numpy as np
    import torch
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]
    import bench
    import hertz_cases as HC
    import hertz_spheres as H
    out[rank] = _calib_grad(bench, HC, H, np, rank, world, lambda g: _allreduce(torch, dist, g))
    dist.destroy_process_group()


def _allreduce(torch, dist, g):
    t = torch.tensor(g, dtype=torch.float64)
    dist.all_reduce(t)
    return t.numpy()


def _calib_grad(bench, HC, H, np, rank, world, reduce):
    scenes, per, steps = 4, 27, 30
    c = HC.gas(seed=9, scenes=scenes)
    lo, hi = bench.rank_range(scenes, rank, world)
    sl = slice(lo * per, hi * per)
    model = H.Model(c["r"][sl], c["m"][sl], c["I"][sl], np.arange(hi - lo + 1) * per, c["planes"], HC.NU, HC.DT,
                    c["g"])
    target = c["x0"][sl] + 1e-5
    tans = [{"theta": np.eye(3)[k]} for k in range(3)]
    x, _, _ = H.jvp(model, c["x0"][sl], c["v0"][sl], c["w0"][sl], HC.THETA, tans, steps)
    # dL/dtheta_k of L = sum ||x - target||^2 / n_all over this rank's scenes
    g = (2.0 * (x.v - target)[..., None] * x.d).sum((0, 1)) / (scenes * per)
    return reduce(g)


def test_calibration_gradient_allreduce_matches_single_rank():
    import numpy as np
    sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]
    import bench
    import hertz_cases as HC
    import hertz_spheres as H
    single = _calib_grad(bench, HC, H, np, 0, 1, lambda g: g)
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_calib_worker, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert np.all(np.abs(single) > 0)
    for rank in range(2):  # every rank holds the whole job's gradient after the all-reduce
        np.testing.assert_allclose(res[rank], single, rtol=1e-12, atol=0)


def _batch_worker(rank, world, port, out):
    """One rank of the batched split: its scenes (split_scenes by body count), each stepped alone by
    the oracle in float and in double, the largest position difference gathered as a max."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "tests"), os.path.join(ROOT, "peclet-dem_b200")]
    import bench
    mine, err = _batch_errors(bench, rank, world)
    out[rank] = (mine, bench.max_over_ranks(err, dist, "cpu"))
    dist.destroy_process_group()


def _batch_scenes():
    import scenes as S
    return [S.dense_spheres(seed=20 + k, n=n, box=((0, 0, 0), (5e-3, 5e-3, 5e-3)))
            for k, n in enumerate((60, 25, 40, 30, 50))]


def _batch_errors(bench, rank, world):
    import numpy as np
    import parity as P
    from peclet.dem._capi import CApi
    orc = CApi(os.path.join(ROOT, "oracle", "_build", "liborc.so"), "orc")
    scs = _batch_scenes()
    mine = bench.split_scenes([sc.n for sc in scs], world)[rank]
    err = 0.0
    for s in mine:
        sc = scs[s]
        a, b = P.build(orc, sc, None, "fp32"), P.build(orc, sc, None, "fp64")
        for _ in range(3):
            a.step(sc.dt)
            b.step(sc.dt)
        err = max(err, float((np.linalg.norm(a.get_positions() - b.get_positions(), axis=1) / sc.global_scale).max()))
    return mine, err


def test_batched_split_error_gather_matches_single_rank(orc_api):
    sys.path[:0] = [ROOT, os.path.join(ROOT, "tests")]
    import bench
    _, single = _batch_errors(bench, 0, 1)
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_batch_worker, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert sorted(res[0][0] + res[1][0]) == list(range(len(_batch_scenes())))
    assert single > 0
    assert res[0][1] == res[1][1] == single


def test_reference_arm_loads_no_library_of_this_repository():
    """The reference arm runs the reference's own build on the headline restart and maps no
    library of this repository (libpdem.so, the scene generator)."""
    code = ("import sys, types; sys.argv=['bench.py']; sys.path.insert(0, %r); import bench; "
            "a = types.SimpleNamespace(steps=1, warmup=0, gpus=1); bench.run_reference_arm(a); "
            "maps = open('/proc/self/maps').read(); "
            "bad = [m for m in ('libpdem', 'librsa', 'liborc') if m in maps]; "
            "assert not bad, bad; assert 'peclet.dem' not in sys.modules; print('clean')") % ROOT
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_omp.so")):
        pytest.skip("reference build (oracle/_ref) not present")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, OMP_NUM_THREADS="2"))
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip().splitlines()[-1] == "clean"
    import json
    line = json.loads(r.stdout.strip().splitlines()[0])
    assert line["impl"] == "reference" and line["config"]["workload"] == "plain_settling_4096_fp64"
