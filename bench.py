"""Benchmark: particle-substeps/s of the plain FP64 XPBD substep on one B200.

Workload (seeded synthetic, no dataset): 262,144 polydisperse spheres, radii lognormal (median
1 mm, sigma 0.25, clipped to [0.5, 2] mm), placed without overlap by random sequential addition in a
box periodic in x and y (L_x = L_y, height 2 L_x, solids fraction 0.35) with a floor plane at z = 0;
density 2500 kg/m^3, e = 0.6, mu = 0.4, gravity -9.81 m/s^2, dt = 2e-5 s split into 10 substeps
(one `step(2e-6)` call = one substep), 10 position and 10 velocity iterations. One benchmark step
= one outer step = 10 substeps. Metric = N x substeps / second.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is device time (two CUDA events on the library's stream around all timed substeps, idle
gaps included; a second pass with per-stage events gives the stage breakdown) with the state
resident in HBM; `e2e` runs the same loop through the public API with host buffers
(external forces copied in, positions and velocities copied out every outer step) timed by the
host clock. `--impl reference` times the reference's own code (its headers built against the
OpenMP flavour of the Kokkos shim) on this machine's host cores. More than one GPU runs replicas
(the single-scene step has no shard-parallel decomposition).

The `batched` object of the line measures the batched form on 512 rotating drums
(`workloads.rotating_drums`, about 1.9 M bodies, one simulation per GPU; scenes split over the
ranks) in FP64 and in the FP32-mixed form, with the mixed form's position error against the FP64
run after the same substeps. `--drums 0` skips it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "peclet-dem_b200"))

import numpy as np  # noqa: E402

METRIC = "particle-substeps/s"
SUBSTEPS = 10
REF_OMP = os.path.join(ROOT, "oracle", "_ref", "libref_omp.so")
REF_SERIAL = os.path.join(ROOT, "oracle", "_ref", "libref_serial.so")


def workload_desc(n):
    return {"workload": f"polydisperse_{n}_periodic_xy_floor_xpbd",
            "particles": n, "substeps_per_step": SUBSTEPS, "dt_substep": 2e-6,
            "radii": "lognormal median 1 mm sigma 0.25 clipped [0.5,2] mm", "solids_fraction": 0.35,
            "iterations": {"position": 10, "velocity": 10}, "precision": "fp64",
            "l2": "state larger than L2 (no flush needed)"}


def make_scene(n):
    from peclet.dem import workloads as W
    return W.polydisperse(n=n)


# ---------------------------------------------------------------------------------------------
# GPU clocks during the timed region
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(self.index)], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            self.p.wait(timeout=10)

    def summary(self):
        self.f.flush()
        self.f.seek(0)
        rows = [r.strip().split(", ") for r in self.f.read().splitlines() if r.strip()]
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for k, name in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------------------------
# algorithmic bytes of one substep (FP64: D = 8 bytes per real) — byte model of the substep:
# particles 81 D N, pairs 16 P, contacts 2 C (8 + 16 D), manifolds M (12 + 20 D), colouring
# 12 (M + C), ledger M (16 + 8 D), velocity sweeps I_v M (12 + 20 D + 53 D), position sweeps
# I_p C (8 + 48 D)
def substep_bytes(n, P, C, M, iv, ip, D=8):
    Sm = 12 + 20 * D
    return (81 * D * n + 16 * P + 2 * C * (8 + 16 * D) + M * Sm + 12 * (M + C) + M * (16 + 8 * D)
            + iv * M * (Sm + 53 * D) + ip * C * (8 + 48 * D))


# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum summed over a stage's kernels in one
# ncu capture of one substep) at the default workload of 262,144 spheres, in bytes per substep;
# stages and sizes not captured report none. The colouring stage covers both colourings with both
# colour orders (one launch) and the manifold incidence lists.
STAGE_DRAM_BYTES = {(262144, "colour_velocity"): 23.0e6}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def max_over_ranks(value, dist=None, device="cpu"):
    """Largest per-rank value over the process group (the device time of the slowest replica).
    NCCL on GPUs; the multi-rank tests run it over gloo on CPU."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world, n, substeps, steps, t_max):
    """Whole-job particle-substeps/s: every replica's work over the slowest replica's time."""
    return world * n * substeps * steps / t_max


def split_scenes(sizes, world):
    """Scenes of the batched form per rank: largest first to the rank with the fewest bodies."""
    loads = [0] * world
    owner = [0] * len(sizes)
    for s in sorted(range(len(sizes)), key=lambda k: -sizes[k]):
        r = min(range(world), key=lambda k: loads[k])
        owner[s] = r
        loads[r] += sizes[s]
    return [[s for s in range(len(sizes)) if owner[s] == r] for r in range(world)]


def run_batched(args, rank, world, dist, dem):
    """Batched rotating drums (512 scenes) in one simulation per GPU, in FP64 and in the FP32-mixed
    form; scenes are split over the ranks with no exchange while stepping. The mixed form's error
    is its largest position difference from the FP64 run after the same substeps, in radii.
    Returns the sub-object of the JSON line."""
    from peclet.dem import workloads as W
    from peclet.dem.batch import apply_batch
    scenes, extras = W.rotating_drums(scenes=args.drums)
    mine = split_scenes([sc.n for sc in scenes], world)[rank]
    sc_m = [scenes[s] for s in mine]
    n_all = sum(sc.n for sc in scenes)
    n_mine = sum(sc.n for sc in sc_m)
    radius = np.concatenate([sc.scales * sc.global_scale for sc in sc_m])
    dt = sc_m[0].dt

    def one(precision):
        sim = dem.Simulation(n_mine + 8, precision)
        apply_batch(sim, sc_m, [extras[s] for s in mine])
        for _ in range(args.warmup * SUBSTEPS):
            sim.step(dt)
        if dist is not None:
            dist.barrier()
        sim.timer_start()
        for _ in range(args.steps * SUBSTEPS):
            sim.step(dt)
        t = max_over_ranks(sim.timer_stop() / 1e3, dist, "cuda")
        sweeps = sim.scene_counters()
        tune = sim.scene_block()  # settled during the warm-up substeps
        x = sim.get_positions()  # the error is measured at the end of the timed substeps
        sim.profile_enable(True)
        for _ in range(args.steps * SUBSTEPS):
            sim.step(dt)
        stages, launches = sim.profile_read()
        sim.profile_enable(False)
        sim.close()
        per_step = {k: round(ms / args.steps, 3) for k, (ms, c) in stages.items() if c}
        return t, per_step, launches, sweeps, x, tune

    t64, st64, l64, sw64, x64, tu64 = one("fp64")
    tmx, stmx, lmx, _, xmx, tumx = one("mixed")
    err = np.linalg.norm(xmx - x64, axis=1) / radius
    err_max = max_over_ranks(float(err.max()) if err.size else 0.0, dist, "cuda")
    rate = lambda t: n_all * SUBSTEPS * args.steps / t
    return {"workload": f"rotating_drums_{len(scenes)}_scenes", "scenes": len(scenes), "particles": n_all,
            "unit": METRIC, "scaling": "weak (scenes split over ranks)",
            "fp64": {"value": rate(t64), "ms_per_step": 1e3 * t64 / args.steps, "gpu_launches": l64,
                     "stages_ms_per_step": st64, "err_vs_fp64": 0.0, "autotuned_scene_block": tu64},
            "mixed": {"value": rate(tmx), "ms_per_step": 1e3 * tmx / args.steps, "gpu_launches": lmx,
                      "stages_ms_per_step": stmx, "autotuned_scene_block": tumx,
                      "err_vs_fp64": {"max_position_error_radii": err_max,
                                      "median_position_error_radii": float(np.median(err)) if err.size else 0.0,
                                      "after_substeps": (args.warmup + args.steps) * SUBSTEPS}},
            "mean_sweeps_last_substep": {"velocity": float(sw64[:, 2].mean()), "position": float(sw64[:, 4].mean())},
            "config": "R 50 mm, L 20 mm drums, omega U[0.5,3] rad/s, N_s U{256..8192} capped at 30% fill of the "
                      "lower half, radii U[0.8,1.2] mm, mu U[0.2,0.8], e U[0.3,0.9], dt 5e-5 s / 10 substeps"}


def run_calibration(args, rank, world, dist):
    """Differentiable calibration: boxes of 2048 spheres (r 1 mm, 40 x 40 x 80 mm, six planes),
    2000 Hertz substeps of 2e-5 s with checkpoints every 100, loss = mean squared distance of the
    final positions to targets made by the same solver at hidden (E, e, mu) = (5e6, 0.7, 0.35);
    gradients with respect to (E, e, mu) and the initial velocities from the adjoint, at the guess
    (4e6, 0.6, 0.3). Scenes are split over ranks; the three material gradients are summed over
    ranks with one all-reduce per backward pass. Reports forward-only and forward+adjoint rates
    (device time, max over ranks), their cost ratio, the gradients' relative error against
    central finite differences (relative steps 1e-4 and 1e-6, FP64) and against the tangent-linear
    (forward-mode dual-number) run along one direction, and the FP32 gradients' error against
    FP64. Returns the sub-object of the JSON line."""
    import torch
    from peclet.dem import workloads as W
    from peclet.dem.adjoint import HertzSpheres
    per = 2048
    c = W.calibration_boxes(scenes=args.calib_scenes)
    lo, hi = (args.calib_scenes * rank) // world, (args.calib_scenes * (rank + 1)) // world
    sl = slice(lo * per, hi * per)
    n_all, n = args.calib_scenes * per, (hi - lo) * per
    steps, ck, dt = args.calib_substeps, 100, 2e-5
    hidden, guess = (5e6, 0.7, 0.35), (4e6, 0.6, 0.3)
    dev = torch.device("cuda", torch.cuda.current_device())

    def make(prec):
        return HertzSpheres(c["r"][sl], c["m"][sl], c["I"][sl], np.arange(hi - lo + 1) * per, c["planes"], 0.3, dt,
                            (0.0, 0.0, -9.81), prec, ck)

    def timed(fn):
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        out = fn()
        b.record()
        torch.cuda.synchronize()
        return out, max_over_ranks(a.elapsed_time(b) / 1e3, dist, "cuda")

    x0 = torch.as_tensor(c["x0"][sl], device=dev)
    v0 = torch.as_tensor(c["v0"][sl], device=dev)
    w0 = torch.as_tensor(c["w0"][sl], device=dev)
    s64 = make("fp64")
    (xt, _, _), _ = s64.run(x0, v0, w0, hidden, steps)  # targets at the hidden parameters

    def loss_of(sim, theta, target, nsteps, vv=None):
        (x, _, _), _ = sim.run(x0, v0 if vv is None else vv, w0, tuple(theta), nsteps)
        part = ((x.double() - target) ** 2).sum()
        if dist is not None:
            dist.all_reduce(part)
        return float(part) / n_all

    def fwd_adj(sim, target, nsteps):
        th = torch.tensor(guess, dtype=torch.float64, requires_grad=True)
        vr = v0.to(sim.dtype).clone().requires_grad_(True)
        x, _, _ = sim.rollout(x0.to(sim.dtype), vr, w0.to(sim.dtype), th, nsteps)
        loss = ((x.double() - target) ** 2).sum() / n_all
        loss.backward()
        g = th.grad.to(dev)
        if dist is not None:
            dist.all_reduce(g)  # the one exchange step: dL/d(E, e, mu) summed over ranks
        return g.cpu().numpy(), vr.grad.double()

    def ranks_sum(x):
        if dist is None:
            return float(x)
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        dist.all_reduce(t)
        return float(t)

    rel = lambda a, b: abs(a - b) / abs(b) if b else None
    gen = torch.Generator(device="cpu").manual_seed(5)
    dv = torch.randn(v0.shape, generator=gen, dtype=torch.float64).to(dev)
    dth = np.array([1e5, 0.01, 0.01])

    def checks(nsteps, target, g64, gv64, g32, gv32):
        """Gradients at one horizon against central finite differences of the FP64 forward
        (relative steps 1e-4 and 1e-6), the directional derivative against the tangent-linear
        run and FD, and the FP32 gradients against FP64."""
        fd = {}
        for rstep in (1e-4, 1e-6):
            row = []
            for k in range(3):
                h = rstep * guess[k]
                tp, tm = list(guess), list(guess)
                tp[k] += h
                tm[k] -= h
                row.append((loss_of(s64, tp, target, nsteps) - loss_of(s64, tm, target, nsteps)) / (2 * h))
            fd[rstep] = row
        got = ranks_sum((gv64 * dv).sum()) + float((g64 * dth).sum())
        h = 1e-4 * 0.2  # relative step 1e-4 of the largest initial speed component
        fd_dir = (loss_of(s64, np.array(guess) + h * dth, target, nsteps, v0 + h * dv)
                  - loss_of(s64, np.array(guess) - h * dth, target, nsteps, v0 - h * dv)) / (2 * h)
        ((xj, _, _), (xdj, _, _)), t_j = timed(lambda: s64.jvp(x0, v0, w0, guess, torch.zeros_like(x0), dv,
                                                              torch.zeros_like(w0), dth, nsteps))
        jv = ranks_sum((2.0 * (xj - target) * xdj).sum()) / n_all
        return {"substeps": nsteps,
                "grad_fp64": {"E": float(g64[0]), "e": float(g64[1]), "mu": float(g64[2])},
                "fd_fp64": {str(r): {"E": v[0], "e": v[1], "mu": v[2]} for r, v in fd.items()},
                "rel_err_vs_fd": {str(r): {"E": rel(g64[0], v[0]), "e": rel(g64[1], v[1]), "mu": rel(g64[2], v[2])}
                                  for r, v in fd.items()},
                "direction": {"adjoint": got, "tangent_linear": jv, "rel_err_vs_tangent_linear": rel(got, jv),
                              "fd_rel_step_1e-4": fd_dir, "rel_err_vs_fd": rel(got, fd_dir),
                              "ms_tangent_linear": 1e3 * t_j,
                              "what": "theta (1e5, 0.01, 0.01) and v0 ~ N(0, 1) per component"},
                "fp32_rel_err_vs_fp64": {"E_e_mu": [float(abs(a - b) / abs(b)) for a, b in zip(g32, g64)],
                                         "v0_rms": float((gv32 - gv64).norm() / gv64.norm()),
                                         "v0_max_abs_over_scale": float((gv32 - gv64).abs().max()
                                                                        / gv64.abs().max())}}

    out = {}
    grads = {}
    s32 = make("fp32")
    for prec, sim in (("fp64", s64), ("fp32", s32)):
        fwd_adj(sim, xt, min(steps, 2 * ck))  # warm-up: allocator, module loading, first launches
        _, t_f = timed(lambda: sim.run(x0, v0, w0, guess, steps))
        (g, gv), t_fa = timed(lambda: fwd_adj(sim, xt, steps))
        grads[prec] = (g, gv)
        out[prec] = {"forward": n_all * steps / t_f, "fwd_adjoint": n_all * steps / t_fa, "cost_ratio": t_fa / t_f,
                     "ms_forward": 1e3 * t_f, "ms_fwd_adjoint": 1e3 * t_fa}
    full = checks(steps, xt, *grads["fp64"], *grads["fp32"])
    # the same checks on a 64-substep horizon (few contacts begin or end inside it)
    short = min(64, steps)
    (xs, _, _), _ = s64.run(x0, v0, w0, hidden, short)
    window = checks(short, xs, *fwd_adj(s64, xs, short), *fwd_adj(s32, xs, short))
    return {"workload": f"calibration_boxes_{args.calib_scenes}x{per}", "particles": n_all, "substeps": steps,
            "checkpoint_every": ck, "unit": METRIC, "scaling": "weak (scenes split over ranks)",
            "path": "step_hertz force law (spheres, planes), hand-written adjoint",
            "fp64": out["fp64"], "fp32": out["fp32"],
            "checks_full_horizon": full, "checks_64_substeps": window, "checkpoints_per_rollout": -(-steps // ck),
            "contact_list_every": s64.list_every, "window_reruns": s64.stats["reruns"],
            "loss_at_guess": loss_of(s64, guess, xt, steps),
            "config": "64 scenes x 2048 spheres r 1 mm, box 40x40x80 mm (6 planes), lattice 8x8x32 + jitter 0.1 mm, "
                      "v U(+-0.2) m/s, E 5e6 Pa hidden / 4e6 guess, e 0.7 / 0.6, mu 0.35 / 0.3, nu 0.3, dt 2e-5 s"}


def run_config_lines(args, dem):
    """Throughput of the other named configurations on this GPU (device time over CUDA events on
    the library's stream, state resident, after warm-up), each as particle-substeps/s:
    - plain XPBD settling, 4,096 spheres, FP64, with the reference's own OpenMP build on the same
      scene beside it (a bounded sample);
    - the Hertz engine on the polydisperse packing (262,144 spheres), closed variant (the
      reference's engine refuses periodic domains and planes: floor and sides are one SDF grid
      wall), FP64 and FP32;
    - 65,536 point-shell hollow cylinders with a 512-point stratified shell, FP64 and the
      FP32-mixed form (box scaled so the bodies can be placed; see workloads.hollow_cylinders)."""
    from peclet.dem import workloads as W

    def timed(sim, one, steps, warm):
        for _ in range(warm):
            one()
        sim.timer_start()
        for _ in range(steps):
            one()
        return sim.timer_stop() / 1e3

    out = {}
    sc = W.plain_settling()
    sim = sc.apply(dem.Simulation(sc.n + 8, "fp64"))
    steps = 100
    t = timed(sim, lambda: [sim.step(sc.dt) for _ in range(sc.substeps)], steps, 3)
    line = {"workload": f"plain_settling_{sc.n}", "unit": METRIC, "dtype": "f64",
            "value": sc.n * sc.substeps * steps / t, "ms_per_step": 1e3 * t / steps,
            "substeps_timed": steps * sc.substeps, "contacts_last_substep": sim.num_contacts()}
    # the working set fits in L2 (126 MB): the byte model's bandwidth is L2 context, not an HBM
    # fraction (counts of the last substep stand for every timed substep)
    c = sim.counters()
    nb = sim.num_particles()
    per_sub = substep_bytes(nb, c["pairs"], c["contacts"], c["manifolds"], c["velocity_sweeps"],
                            c["position_sweeps"])
    line["l2_resident"] = {
        "working_set_mb": round((nb * 300 + c["pairs"] * 8 + c["contacts"] * 2 * (8 + 16 * 8)
                                 + c["manifolds"] * (12 + 20 * 8)) / 1e6, 2),
        "algorithmic_gbps": per_sub * sc.substeps * steps / t / 1e9,
        "counts_last_substep": {k: c[k] for k in ("pairs", "contacts", "manifolds", "velocity_sweeps",
                                                  "position_sweeps")}}
    sim.close()
    if not args.no_cpu and os.path.exists(REF_OMP):
        threads = os.cpu_count() or 1
        v, el = cpu_reference(sc, 200, threads)
        line["cpu_reference"] = {"value": v, "unit": METRIC, "cores": threads, "kind": "reference",
                                 "sample": f"200 substeps of the same scene, {el:.1f} s"}
    if not args.no_cpu and os.path.exists(REF_SERIAL):
        v, el = cpu_reference(sc, 100, 1, REF_SERIAL)
        line["cpu_reference_serial"] = {"value": v, "unit": METRIC, "cores": 1, "kind": "reference",
                                        "sample": f"100 substeps of the same scene, serial shim build, "
                                                  f"{el:.1f} s"}
    out["settling"] = line

    sc, extra = W.polydisperse_hertz_closed()
    line = {"workload": f"polydisperse_{sc.n}_closed_hertz", "unit": METRIC}
    for prec in ("fp64", "fp32"):
        sim = sc.apply(dem.Simulation(sc.n + 8, prec))
        extra(sim)
        steps = 5
        t = timed(sim, lambda: sim.step_hertz(sc.dt, sc.substeps, 0.3), steps, 2)
        line[prec] = {"value": sc.n * sc.substeps * steps / t, "ms_per_step": 1e3 * t / steps,
                      "substeps_timed": steps * sc.substeps}
        sim.close()
    out["hertz"] = line

    sc = W.hollow_cylinders(shell_points=W.hollow_cylinder_shell())
    line = {"workload": f"hollow_cylinders_{sc.n}_shell512", "unit": METRIC,
            "box_m": [float(v) for v in sc.domain[1]]}
    for prec in ("fp64", "mixed"):
        sim = sc.apply(dem.Simulation(sc.n + 8, prec))
        steps = 3
        t = timed(sim, lambda: [sim.step(sc.dt) for _ in range(sc.substeps)], steps, 1)
        line[prec] = {"value": sc.n * sc.substeps * steps / t, "ms_per_step": 1e3 * t / steps,
                      "substeps_timed": steps * sc.substeps, "contacts_last_substep": sim.num_contacts()}
        if prec == "fp64":
            x64 = sim.get_positions()
        else:
            err = np.linalg.norm(sim.get_positions() - x64, axis=1) / sc.global_scale
            line[prec]["err_vs_fp64"] = {"max_position_error_radii": float(err.max()),
                                         "median_position_error_radii": float(np.median(err)),
                                         "after_substeps": (steps + 1) * sc.substeps}
        sim.close()
    out["shells"] = line
    return out


# ---------------------------------------------------------------------------------------------
def cpu_reference(scene, substeps, threads, lib=REF_OMP):
    """Time the reference's own substep (OpenMP shim build, or the serial one) for `substeps`
    calls; returns particle-substeps/s. State set exactly as on the GPU (the reference computes in
    float)."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    os.environ.setdefault("OMP_PROC_BIND", "close")
    from peclet.dem._capi import CApi, CApiSimulation
    api = CApi(lib, "ref")
    sim = scene.apply(CApiSimulation(api, scene.n + 8, "fp32"))
    sim.step(scene.dt)  # warm-up: first-touch allocations and ghost capacity
    t = time.perf_counter()
    for _ in range(substeps):
        sim.step(scene.dt)
    dt = time.perf_counter() - t
    sim.close()
    return scene.n * substeps / dt, dt


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if not os.path.exists(REF_OMP):
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/libref_omp.so missing"}))
        return 0
    threads = os.cpu_count() or 1
    scene = make_scene(args.particles)
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from peclet.dem._capi import CApi, CApiSimulation
    api = CApi(REF_OMP, "ref")
    sim = scene.apply(CApiSimulation(api, scene.n + 8, "fp32"))
    # one reference "step" = one substep of the workload (a bounded sample: an outer step of 10
    # substeps at this size takes tens of seconds on the host)
    for _ in range(args.warmup):
        sim.step(scene.dt)
    t = time.perf_counter()
    for _ in range(args.steps):
        sim.step(scene.dt)
    el = time.perf_counter() - t
    value = scene.n * args.steps / el
    cfg = workload_desc(scene.n)
    cfg["precision"] = "fp32 (the reference computes in float)"
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": cfg, "impl": "reference",
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "reference",
                         "sample": f"{args.steps} substeps of the {scene.n}-sphere workload after "
                                   f"{args.warmup} warm-up substeps; OpenMP, {threads} threads"},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
    return 0


def run_ours(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    import peclet.dem as dem
    from peclet.dem._capi import STAGES
    dem._API.check(dem._API.fn["set_device"](local), "set_device")

    scene = make_scene(args.particles)
    n = scene.n
    sim = scene.apply(dem.Simulation(n + 8, "fp64"))
    # the configuration runs 200 steps from rest; the timed steps sit in its middle (after
    # `--presettle` untimed steps), where the first spheres reach the floor
    for _ in range(args.presettle + args.warmup):
        for _ in range(SUBSTEPS):
            sim.step(scene.dt)

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- device-timed region ----
    clocks = ClockSampler(local)
    with clocks:
        time.sleep(0.5)  # sampler running before the timed region starts
        barrier()
        timed_allocs = dem._API.fn["debug_allocs"]()
        t0 = time.perf_counter()
        sim.timer_start()  # events on the library's stream around the whole timed region
        for _ in range(args.steps):
            for _ in range(SUBSTEPS):
                sim.step(scene.dt)
        dev_ms = sim.timer_stop()
        wall = time.perf_counter() - t0
        timed_allocs = dem._API.fn["debug_allocs"]() - timed_allocs
    barrier()
    # the same number of steps again with per-stage events (their synchronisation per substep
    # slows the step; these figures explain the timed value, they are not it)
    sim.profile_enable(True)
    for _ in range(args.steps):
        for _ in range(SUBSTEPS):
            sim.step(scene.dt)
    stages, launches = sim.profile_read()
    counts = sim.debug_counts()
    sweeps = sim.debug_sweeps() if hasattr(sim, "debug_sweeps") else None
    reuse = sim.debug_reuse()
    last = sim.counters()
    sim.profile_enable(False)
    # max over ranks of the device time; value = all ranks' particle-substeps / that time
    t_max = max_over_ranks(dev_ms / 1e3, dist, "cuda")
    value = aggregate_rate(world, n, SUBSTEPS, args.steps, t_max)

    # ---- end to end through the public API with host buffers (pinned, as a data loader's) ----
    import torch
    pinned = lambda: torch.zeros((n, 3), dtype=torch.float64, pin_memory=True).numpy()
    force, pos, vel = pinned(), pinned(), pinned()
    barrier()
    te = time.perf_counter()
    allocs = dem._API.fn["debug_allocs"]
    a0 = allocs()
    laps = []
    for _ in range(args.steps):
        tl = time.perf_counter()
        sim.set_external_forces(force)
        for _ in range(SUBSTEPS):
            sim.step(scene.dt)
        sim.get_positions(out=pos)
        sim.get_velocities(out=vel)
        laps.append(round(1e3 * (time.perf_counter() - tl), 2))
    e2e_s = time.perf_counter() - te
    assert np.all(np.isfinite(pos)) and np.all(np.isfinite(vel))
    e2e = {"value": world * n * SUBSTEPS * args.steps / e2e_s, "unit": METRIC,
           "h2d_bytes_per_step": int(force.nbytes), "d2h_bytes_per_step": int(pos.nbytes + vel.nbytes),
           "ms_per_step_each": laps, "device_allocations": int(allocs() - a0)}

    # ---- roofline of the dominant stage ----
    per_step = {k: (ms / args.steps, c / args.steps) for k, (ms, c) in stages.items() if c}
    peak, peak_kind = measured_peaks()
    P, C, M = counts["pairs"], counts["contacts"], counts["manifolds"]
    iv = sweeps["velocity"] / args.steps / SUBSTEPS if sweeps else 10
    ip = sweeps["position"] / args.steps / SUBSTEPS if sweeps else 10
    stage_bytes = {
        "velocity": iv * M * (12 + 20 * 8 + 53 * 8),
        "position": ip * C * (8 + 48 * 8),
        "broadphase": n * 4 * 8 + 8 * P,
        "narrowphase": 8 * P + C * (8 + 16 * 8),
        "manifolds": 2 * C * (8 + 16 * 8) + M * (12 + 20 * 8),
        "colour_velocity": 12 * (M + C),
        "ledger": M * (16 + 8 * 8),
    }
    step_bytes = substep_bytes(n, P, C, M, iv, ip) * SUBSTEPS
    # the dominant stage among those with a byte model (all the heavy ones)
    roof_stage = max((k for k in per_step if k in stage_bytes), key=lambda k: per_step[k][0])
    st_ms = per_step[roof_stage][0] / SUBSTEPS
    achieved = stage_bytes[roof_stage] / (st_ms / 1e3) / 1e9 if st_ms > 0 else 0.0
    traffic = STAGE_DRAM_BYTES.get((n, roof_stage))
    roofline = {"bound": "hbm", "kernel": f"{roof_stage} stage (per substep)", "achieved": achieved,
                "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": traffic, "traffic_unit": "bytes per substep (ncu)",
                "algorithmic_bytes": stage_bytes[roof_stage],
                "step_algorithmic_GBps": step_bytes / (dev_ms / 1e3 / args.steps) / 1e9}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu and os.path.exists(REF_OMP):
        threads = os.cpu_count() or 1
        v, el = cpu_reference(scene, args.cpu_substeps, threads)
        cpu = {"value": v, "unit": METRIC, "cores": threads, "kind": "reference",
               "sample": f"{args.cpu_substeps} substeps of the same {n}-sphere workload (reference code, "
                         f"OpenMP Kokkos-shim build, float), {el:.1f} s"}

    batched = run_batched(args, rank, world, dist, dem) if args.drums > 0 else None
    calib = run_calibration(args, rank, world, dist) if args.calib_scenes > 0 else None
    configs = run_config_lines(args, dem) if (rank == 0 and not args.no_configs) else None

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": dict(workload_desc(n), parallelism="replicas" if world > 1 else "single",
                           timed_steps_from=args.presettle + args.warmup),
            "e2e": e2e, "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu,
            "clocks": clocks.summary(), "wall_ms_per_step": 1e3 * wall / args.steps,
            "stages_ms_per_step": {k: round(v[0], 4) for k, v in per_step.items()},
            "counts_last_substep": counts, "sweeps": sweeps, "topology_kept": reuse, "last_substep": last, "batched": batched,
            "fwd_adjoint": calib, "configs": configs,
            "device_allocations_timed": int(timed_allocs),
        }
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--particles", type=int, default=262144)
    ap.add_argument("--cpu-substeps", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--drums", type=int, default=512, help="scenes of the batched line (0: skip it)")
    ap.add_argument("--calib-scenes", type=int, default=64, help="scenes of the calibration line (0: skip it)")
    ap.add_argument("--calib-substeps", type=int, default=2000)
    ap.add_argument("--no-configs", action="store_true", help="skip the settling / Hertz / shell lines")
    ap.add_argument("--presettle", type=int, default=95,
                    help="untimed steps of the 200-step run before the warm-up and timed steps")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
