"""GPU parity at the benchmark configurations' scales, through the C ABI, against the oracle
restatement: bit-exact at float, within 1e-12 relative at double, after every substep or call.

* the 4,096-sphere settling configuration restarted from its saved settled state (the
  benchmark's own window: 12.4k manifolds in 8-12 colours, every sweep loop at full length, the
  stabilization pass and the support levels every substep; these sizes take the one-cluster and
  cooperative sweep paths that the small parity scenes do not reach);
* 8,192 polydisperse spheres in a box periodic in x and y (the polydisperse generator, about 1,700
  ghost images), with random velocities;
* 256 hollow cylinders with the 512-point stratified shell, placed overlapping (about 20k contacts);
* the closed Hertz variant of the polydisperse packing at 16,384 spheres, with random velocities,
  two calls of 10 substeps (tangential history included).
"""
import numpy as np
import pytest

import parity as P
import scenes as S
from peclet.dem import workloads as W

pytestmark = pytest.mark.gpu


def _settled():
    return W.plain_settled()


def _periodic8k():
    sc = W.polydisperse(n=8192, seed=6)
    sc.vel = np.random.default_rng(6).uniform(-0.5, 0.5, sc.pos.shape)
    sc.dt = 1e-5
    return sc


def _shells256():
    return S.cylinders(seed=41, n=256, L=20e-3, shell=W.hollow_cylinder_shell())


CASES = [("settled_4096_restart", _settled, 10), ("periodic_polydisperse_8192", _periodic8k, 6),
         ("shells_256_x512", _shells256, 4)]


@pytest.mark.parametrize("precision,rtol", [("fp32", 0.0), ("fp64", 1e-12)])
@pytest.mark.parametrize("name,mk,steps", CASES, ids=[c[0] for c in CASES])
def test_config_scale_vs_oracle(gpu_api, orc_api, name, mk, steps, precision, rtol):
    sc = mk()
    a = P.build(gpu_api, sc, None, precision)
    b = P.build(orc_api, sc, None, precision)
    for k in range(steps):
        a.step(sc.dt)
        b.step(sc.dt)
        bad = P.diff(P.snapshot(a), P.snapshot(b), rtol=rtol)
        assert not bad, f"{name} {precision}: substep {k}: {bad[:4]}"
    c = a.counters()
    assert c["status"] == 0 and c["contacts"] > 0


@pytest.mark.parametrize("precision,rtol", [("fp32", 0.0), ("fp64", 1e-12)])
def test_hertz_closed_16k_vs_oracle(gpu_api, orc_api, precision, rtol):
    sc, extra = W.polydisperse_hertz_closed(n=16384)
    sc.vel = np.random.default_rng(7).uniform(-3.0, 3.0, sc.pos.shape)
    a = P.build(gpu_api, sc, extra, precision)
    b = P.build(orc_api, sc, extra, precision)
    for k in range(2):
        a.step_hertz(sc.dt, sc.substeps, 0.3)
        b.step_hertz(sc.dt, sc.substeps, 0.3)
        sa, sb = P.snapshot(a, products=False), P.snapshot(b, products=False)
        ka, xa = a.debug_hertz()
        kb, xb = b.debug_hertz()
        sa.update(hk=ka, hx=xa)
        sb.update(hk=kb, hx=xb)
        bad = P.diff(sa, sb, rtol=rtol)
        assert not bad, f"hertz 16k {precision}: call {k}: {bad[:4]}"
    assert np.count_nonzero(xa) > 0
