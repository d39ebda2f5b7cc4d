"""The batched form on the GPU against each scene stepped alone by the oracle.

Four drums of different sizes, rotation rates, restitution and friction share one simulation
(their bodies concatenated, all of them in the same region of space). After every substep each
scene's slice of the batch must equal the oracle's run of that scene alone: bit-exact at float,
within 1e-12 relative at double, as for the single-scene parity tests."""
import numpy as np
import pytest

import parity as P
import scenes as S
from peclet.dem._capi import CApiSimulation
from peclet.dem.batch import apply_batch

pytestmark = pytest.mark.gpu

SPECS = [(31, 60, 1.0, 0.5, 0.3), (32, 140, 2.5, 0.7, 0.6), (33, 90, 0.5, 0.3, 0.2), (34, 160, 3.0, 0.9, 0.8)]


def _drums():
    return [S.spheres_in_drum(seed=seed, n=n, omega=om, e=e, mu=mu) for seed, n, om, e, mu in SPECS]


@pytest.mark.parametrize("precision,rtol", [("fp32", 0.0), ("fp64", 1e-12)])
def test_batch_matches_each_scene_alone(gpu_api, orc_api, precision, rtol):
    drums = _drums()
    scenes = [d[0] for d in drums]
    batch = CApiSimulation(gpu_api, sum(sc.n for sc in scenes) + 8, precision)
    first = apply_batch(batch, scenes, [d[1] for d in drums])
    alone = [P.build(orc_api, sc, ex, precision) for sc, ex in drums]
    dt = scenes[0].dt
    for k in range(12):
        batch.step(dt)
        for a in alone:
            a.step(dt)
        got = P.snapshot(batch, products=False)
        for s, a in enumerate(alone):
            sl = slice(int(first[s]), int(first[s + 1]))
            mine = {key: v[sl] for key, v in got.items()}
            bad = P.diff(mine, P.snapshot(a, products=False), rtol=rtol)
            assert not bad, f"{precision}: substep {k}, scene {s}: {bad[:4]}"
    assert batch.scene_counters().shape == (len(scenes), 5)


def test_batch_overlap_per_scene(gpu_api, orc_api):
    """Each scene's max overlap is its own (the reference's max_overlap of that scene alone)."""
    drums = _drums()
    scenes = [d[0] for d in drums]
    batch = CApiSimulation(gpu_api, sum(sc.n for sc in scenes) + 8, "fp32")
    apply_batch(batch, scenes, [d[1] for d in drums])
    batch.step(scenes[0].dt)
    got = batch.scene_counters()[:, 0]
    for s, (sc, ex) in enumerate(drums):
        a = P.build(orc_api, sc, ex, "fp32")
        a.step(sc.dt)
        assert got[s] == np.float64(np.float32(a.max_overlap()))


def test_batch_rejects_periodic(gpu_api):
    sc = S.polydisperse_periodic()
    batch = CApiSimulation(gpu_api, 2 * sc.n + 8, "fp64")
    apply_batch(batch, [sc, S.polydisperse_periodic(seed=14)])
    with pytest.raises(RuntimeError):
        batch.step(sc.dt)
