"""GPU parity: the B200 step against the CPU checkers, through the C ABI.

* fp32 B200 vs the reference itself (oracle/_ref, its own headers built against the serial Kokkos
  shim) — bit-exact: candidate pairs, contacts, manifolds, colours, warm-start ledger, support
  levels and the state after every substep;
* fp32 B200 vs the oracle restatement at float — bit-exact (always available);
* fp64 B200 vs the oracle restatement at double — every product and the state within 1e-12
  relative (the FP64 acceptance bar; the implementation is expected to be bit-exact).
"""
import numpy as np
import pytest

import parity as P

pytestmark = pytest.mark.gpu


def _run_pair(api_a, api_b, name, mk, extra, steps, precision, rtol):
    sc = mk()
    a = P.build(api_a, sc, extra, precision)
    b = P.build(api_b, sc, extra, precision)
    for k in range(steps):
        a.step(sc.dt)
        b.step(sc.dt)
        bad = P.diff(P.snapshot(a), P.snapshot(b), rtol=rtol)
        assert not bad, f"{name}: substep {k}: {bad[:4]}"


@pytest.mark.parametrize("name,mk,extra,steps", P.MATRIX, ids=[m[0] for m in P.MATRIX])
def test_fp32_bitexact_vs_oracle(gpu_api, orc_api, name, mk, extra, steps):
    _run_pair(gpu_api, orc_api, name, mk, extra, steps, "fp32", 0.0)


@pytest.mark.parametrize("name,mk,extra,steps", P.MATRIX, ids=[m[0] for m in P.MATRIX])
def test_fp64_vs_oracle(gpu_api, orc_api, name, mk, extra, steps):
    _run_pair(gpu_api, orc_api, name, mk, extra, steps, "fp64", 1e-12)


@pytest.mark.parametrize("name,mk,extra,steps", P.MATRIX[:8], ids=[m[0] for m in P.MATRIX[:8]])
def test_fp32_bitexact_vs_reference(gpu_api, ref_api, name, mk, extra, steps):
    _run_pair(gpu_api, ref_api, name, mk, extra, steps, "fp32", 0.0)


def test_step_n_and_counters(gpu_api):
    """step_n(dt, n) is n calls of step(dt), bit for bit; counters() reports the last substep."""
    import scenes as S
    sc = S.dense_spheres()
    a = P.build(gpu_api, sc, None, "fp32")
    b = P.build(gpu_api, sc, None, "fp32")
    for _ in range(5):
        a.step(sc.dt)
    b.step_n(sc.dt, 5)
    assert not P.diff(P.snapshot(a), P.snapshot(b))
    c = b.counters()
    assert c["contacts"] == b.num_contacts() and c["manifolds"] == b.num_manifolds()
    assert c["pairs"] >= c["manifolds"] > 0
    assert c["colors_velocity"] > 0 and c["colors_position"] > 0
    assert 1 <= c["velocity_sweeps"] <= sc.iterations[1] and 1 <= c["position_sweeps"] <= sc.iterations[0]
    assert c["status"] == 0
    assert c["max_overlap"] == b.max_overlap()
    with pytest.raises(ValueError):
        b.step_n(sc.dt, -1)


def test_device_views(gpu_api):
    """get_*_view alias the simulation's device memory: they equal the getters, and forces written
    into the external-force view drive the next steps exactly as set_external_forces does."""
    import numpy as np
    import scenes as S
    sc = S.dense_spheres()
    for prec in ("fp64", "fp32"):
        a = P.build(gpu_api, sc, None, prec)
        b = P.build(gpu_api, sc, None, prec)
        a.step(sc.dt)
        b.step(sc.dt)
        pv, vv, mv = a.get_positions_view(), a.get_velocities_view(), a.get_inv_mass_view()
        assert pv.shape == (sc.n, 3) and mv.shape == (sc.n,)
        np.testing.assert_array_equal(pv.cpu().numpy(), a.get_positions())
        np.testing.assert_array_equal(vv.cpu().numpy(), a.get_velocities())
        np.testing.assert_array_equal(mv.cpu().numpy().astype(np.float64), np.asarray(sc.inv_mass, dtype=mv.cpu().numpy().dtype))
        f = np.random.default_rng(3).normal(scale=1e-4, size=(sc.n, 3))
        fv = a.get_external_forces_view()
        torch = __import__("torch")
        fv.copy_(torch.as_tensor(f, dtype=fv.dtype, device=fv.device))
        torch.cuda.synchronize()  # the write (on torch's stream) completes before the next step
        b.set_external_forces(f.astype(fv.cpu().numpy().dtype).astype(np.float64))
        for _ in range(3):
            a.step(sc.dt)
            b.step(sc.dt)
        assert not P.diff(P.snapshot(a), P.snapshot(b)), prec


def test_domain_getters(gpu_api, orc_api):
    import scenes as S
    for setup in (lambda s: s.set_domain(0.02, 0.03, 0.04), lambda s: s.set_domain((-1e-3, 0, 2e-3), (5e-3, 6e-3, 7e-3))):
        for prec in ("fp32", "fp64"):
            a = P.build(gpu_api, S.dense_spheres(), setup, prec)
            b = P.build(orc_api, S.dense_spheres(), setup, prec)
            assert (a.get_domain_min(), a.get_domain_max()) == (b.get_domain_min(), b.get_domain_max())


def test_contact_grouping_ranked(gpu_api):
    """The stable key sort of the contact list runs as a rank scatter: the narrowphase's list is in
    key order up to its boundary contacts, so every substep with contacts takes it and none of the
    parity scenes' lists is rejected (the tests above check the product against the oracle)."""
    ranked = 0
    for name, mk, extra, steps in P.MATRIX:
        sc = mk()
        a = P.build(gpu_api, sc, extra, "fp64")
        a.profile_enable(True)
        for _ in range(min(steps, 4)):
            a.step(sc.dt)
        r = a.debug_ranked()
        assert r["rejected"] == 0, name
        ranked += r["ranked"]
    assert ranked > 0


def test_contact_grouping_sorted_path():
    """PDEM_CONTACT_SORT=1 keeps the key sort (the rank scatter's fallback): scenes with ghosts,
    planes, SDF walls and point shells stay bit-exact against the oracle that way."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sel = "test_fp32_bitexact_vs_oracle and (periodic_polydisperse or dense_spheres or drum_sdf_wall or hollow_cylinders or settled_column)"
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-m", "gpu", "-k", sel,
                        os.path.join(root, "tests", "test_gpu_parity.py")],
                       cwd=root, env={**os.environ, "PDEM_CONTACT_SORT": "1"}, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert " passed" in r.stdout and "5 passed" in r.stdout, r.stdout[-500:]


@pytest.mark.parametrize("precision,rtol", [("fp32", 0.0), ("fp64", 1e-12)])
def test_shell_plane_reach_cull(gpu_api, orc_api, precision, rtol):
    """Shell bodies at heights stepping through the plane-reach bound (shell reach plus the contact
    margin), one orientation with a rim corner straight down: the culled boundary probes leave the
    contacts, overlaps and state identical to the oracle's full probing."""
    import scenes as S
    _run_pair(gpu_api, orc_api, "shells_at_floor", S.shells_at_floor, None, 4, precision, rtol)


@pytest.mark.parametrize("tail", ["0", "4096"])
def test_colouring_tail_settings(tail):
    """The colouring's hand-over to one block is a launch-shape setting: with no tail (0) and with
    the global-memory tail (4096, beyond the shared-memory tables) scenes of every kind stay
    bit-exact against the oracle (the default, the shared-memory tail, runs in every test above)."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sel = ("test_fp32_bitexact_vs_oracle and (periodic_polydisperse or dense_spheres or drum_sdf_wall "
           "or hollow_cylinders or settled_column)")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-m", "gpu", "-k", sel,
                        os.path.join(root, "tests", "test_gpu_parity.py")],
                       cwd=root, env={**os.environ, "PDEM_COLOR_TAIL": tail}, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "5 passed" in r.stdout, r.stdout[-500:]


def _restore_bodies(sim, sc):
    """Set the scene's per-body state again (as Scene.apply orders the setters)."""
    sim.set_positions(sc.pos)
    if sc.quat is not None:
        sim.set_quaternions(sc.quat)
    if sc.scales is not None:
        sim.set_scales(sc.scales)
    sim.set_velocities(sc.vel)
    sim.set_inv_mass(sc.inv_mass)
    sim.set_inv_inertia(sc.inv_inertia)


def test_grid_barrier_time_out_reports_and_recovers(gpu_api, orc_api, monkeypatch):
    """A grid-wide barrier wait of the persistent loops that runs out (its poll limit cut to one)
    makes the kernel return and the step report an error, leaving the device usable; with the
    default limit restored and the bodies' state set again, the next substeps match the oracle."""
    import scenes as S
    monkeypatch.setenv("PDEM_SWEEP_CLUSTER_ENTRIES", "0")  # every sweep loop on the cooperative grid
    sc = S.dense_spheres()
    sim = P.build(gpu_api, sc, None, "fp64")
    sim.debug_set_barrier_spins(1)
    with pytest.raises(RuntimeError, match="barrier"):
        for _ in range(3):
            sim.step(sc.dt)
    sim.debug_set_barrier_spins(0)
    _restore_bodies(sim, sc)
    ref = P.build(orc_api, sc, None, "fp64")
    for k in range(4):
        sim.step(sc.dt)
        ref.step(sc.dt)
        bad = P.diff(P.snapshot(sim), P.snapshot(ref), rtol=1e-12)
        assert not bad, f"after the time-out, substep {k}: {bad[:4]}"
    assert sim.counters()["status"] == 0
