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


def _columns():
    """Settling lattice columns: resting contacts under gravity fire the stabilization pass (support
    levels, side flags) in every scene."""
    out = []
    for seed, (e, mu) in zip((41, 42, 43), ((0.5, 0.5), (0.3, 0.8), (0.8, 0.2))):
        sc = S.settled_column(seed=seed)
        sc.material = (e, 0.0, mu)
        out.append((sc, None))
    return out


CASES = [("drums", _drums, 12), ("columns", _columns, 25)]


@pytest.mark.parametrize("precision,rtol", [("fp32", 0.0), ("fp64", 1e-12)])
@pytest.mark.parametrize("name,mk,steps", CASES, ids=[c[0] for c in CASES])
def test_batch_matches_each_scene_alone(gpu_api, orc_api, name, mk, steps, precision, rtol):
    cases = mk()
    scenes = [c[0] for c in cases]
    batch = CApiSimulation(gpu_api, sum(sc.n for sc in scenes) + 8, precision)
    first = apply_batch(batch, scenes, [c[1] for c in cases])
    alone = [P.build(orc_api, sc, ex, precision) for sc, ex in cases]
    dt = scenes[0].dt
    stab = np.zeros(len(scenes))
    for k in range(steps):
        batch.step(dt)
        for a in alone:
            a.step(dt)
        counters = batch.scene_counters()
        assert counters.shape == (len(scenes), 5)
        stab += counters[:, 3]
        got = P.snapshot(batch, products=False)
        got["grounded"] = batch.debug_grounded()  # support levels (stabilization), per body
        for s, a in enumerate(alone):
            sl = slice(int(first[s]), int(first[s + 1]))
            mine = {key: v[sl] for key, v in got.items()}
            want = P.snapshot(a, products=False)
            want["grounded"] = a.debug_grounded()
            bad = P.diff(mine, want, rtol=rtol)
            assert not bad, f"{name} {precision}: substep {k}, scene {s}: {bad[:4]}"
    if name == "columns":
        assert stab.min() > 0, "the stabilization pass (support levels) did not run in every scene"


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


def test_autotuned_block_keeps_results(gpu_api, monkeypatch):
    """The launch shape autotuner cycles block sizes over the first substeps and keeps the fastest;
    the results equal a run with the block fixed (the block size changes no result)."""
    drums = _drums()
    scenes = [d[0] for d in drums]
    runs = []
    for fixed in (None, "64"):
        if fixed:
            monkeypatch.setenv("PDEM_SCENE_BLOCK", fixed)
        else:
            monkeypatch.delenv("PDEM_SCENE_BLOCK", raising=False)
        batch = CApiSimulation(gpu_api, sum(sc.n for sc in scenes) + 8, "fp32")
        apply_batch(batch, scenes, [d[1] for d in drums])
        for _ in range(16):
            batch.step(scenes[0].dt)
        runs.append((P.snapshot(batch, products=False), batch.scene_block()))
    (a, ta), (b, tb) = runs
    assert ta["block"] in (64, 128, 256, 512) and all(m > 0 for m in ta["ms"])
    assert tb["block"] == 64
    assert not P.diff(a, b)


def test_autotuned_colour_block_keeps_results(gpu_api, monkeypatch):
    """The batched form also tunes the colouring launch's block (256, 512, 1024, timed over the
    first colourings); the colours do not depend on it, so the run equals one with the block
    fixed. The colourings run on the cooperative grid here (the one-cluster path takes no block)."""
    monkeypatch.setenv("PDEM_COLOR_CLUSTER_ENTRIES", "0")
    drums = _drums()
    scenes = [d[0] for d in drums]
    runs = []
    for fixed in (None, "256"):
        if fixed:
            monkeypatch.setenv("PDEM_COLOR_BLOCK", fixed)
        else:
            monkeypatch.delenv("PDEM_COLOR_BLOCK", raising=False)
        batch = CApiSimulation(gpu_api, sum(sc.n for sc in scenes) + 8, "fp32")
        apply_batch(batch, scenes, [d[1] for d in drums])
        for _ in range(16):
            batch.step(scenes[0].dt)
        runs.append((P.snapshot(batch, products=False), batch.color_block()))
    (a, ta), (b, tb) = runs
    assert ta["block"] in (256, 512, 1024) and all(m > 0 for m in ta["ms"])
    assert tb["block"] == 256
    assert not P.diff(a, b)
