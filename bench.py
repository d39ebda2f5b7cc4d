"""Benchmark: particle-substeps/s of the plain FP64 XPBD substep on one B200.

Headline workload: the plain XPBD settling configuration, 4,096 monodisperse spheres (r 1 mm,
density 2500 kg/m^3, jittered simple-cubic lattice at the bottom of a closed 16 x 16 x 64-cell box
of six planes, e 0.5, mu 0.5, gravity -9.81 m/s^2, 10 position and 10 velocity iterations,
10 substeps of 1e-5 s per outer step, 1,000 outer steps from the lattice start). Both arms restart
from the saved state after 800 of those steps (peclet/dem/states/plain_settling_4096_step800.npz,
made by the FP64 step: the bed is at rest in dense contact, which is where the solve loops run
their full sweeps), run `--warmup` untimed outer steps and then time `--steps` outer steps. One
benchmark step = one outer step = 10 `step(1e-5)` calls. Metric = N x substeps / second.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--extras LIST]

`value`: device time of the K timed outer steps (CUDA events on the library's stream around each
step, summed; L2 flushed between steps by a 256 MiB write, since the 4,096-sphere state fits in
L2). `e2e`: the same window through the public API from the same state, with the external forces
copied in from pinned host memory and positions and velocities copied out every outer step, timed
by the host clock. `--impl reference` times the reference's own code for the path (its headers
built unmodified against the OpenMP flavour of the Kokkos shim, oracle/_ref) on the same state,
the same warm-up and the same timed outer steps, with every host thread; it loads no library of
this repository. More than one GPU runs replicas of the single scene (it does not shard); the
batched drums and calibration scenes are split over the ranks.

Besides the headline, rank 0 prints a detail line first (no "metric" key) with the other
configurations (`--extras`, default all): `xpbd262k` (262,144 polydisperse spheres in a box
periodic in x and y, through the XPBD step: not a configuration the reference names for this
step), `batched` (512 rotating drums after their deposition, FP64 and FP32-mixed), `calibration`
(forward and forward + adjoint of the Hertz rollout), `hertz` (262,144 polydisperse spheres,
closed variant) and `shells` (65,536 hollow cylinders with 512-point shells after a gravity
deposition). The main line, printed last, carries flat keys with their headline figures.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "peclet-dem_b200")
DEM_DIR = os.path.join(PKG_DIR, "peclet", "dem")
sys.path.insert(0, PKG_DIR)

import numpy as np  # noqa: E402

METRIC = "particle-substeps/s"
SUBSTEPS = 10
REF_OMP = os.path.join(ROOT, "oracle", "_ref", "libref_omp.so")         # -march=x86-64-v4
REF_OMP_V2 = os.path.join(ROOT, "oracle", "_ref", "libref_omp_v2.so")   # -march=x86-64-v2 fallback
REF_SERIAL = os.path.join(ROOT, "oracle", "_ref", "libref_serial.so")
# calibration first: it allocates through torch, which later lines' pooled simulation buffers
# would crowd
EXTRAS = ("calibration", "xpbd_adjoint", "xpbd262k", "batched", "hertz", "shells")
L2_FLUSH_BYTES = 256 << 20


def _file_module(name, path):
    """A module loaded from its file alone: no package __init__ runs (the reference arm must not
    load libpdem.so, which importing the peclet.dem package does)."""
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def workloads_module():
    return _file_module("pdem_bench_workloads", os.path.join(DEM_DIR, "workloads.py"))


def capi_module():
    return _file_module("pdem_bench_capi", os.path.join(DEM_DIR, "_capi.py"))


def _cpu_flags():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def ref_omp_lib():
    """The OpenMP reference build for this host: the AVX-512 (x86-64-v4) build when the CPU has
    it, else the x86-64-v2 one. Returns (path, march) or (None, None)."""
    if os.path.exists(REF_OMP) and {"avx512f", "avx512bw", "avx512dq", "avx512vl"} <= _cpu_flags():
        return REF_OMP, "x86-64-v4"
    if os.path.exists(REF_OMP_V2):
        return REF_OMP_V2, "x86-64-v2"
    return None, None


def headline_desc(world=1):
    return {"workload": "plain_settling_4096_fp64", "particles": 4096, "substeps_per_step": SUBSTEPS,
            "dt_substep": 1e-5, "iterations": {"position": 10, "velocity": 10},
            "state": "restart at outer step 800 of 1000 (saved FP64 state), both arms; ledger cold",
            "l2": "flushed between timed steps (256 MiB); state ~4 MB",
            "parallelism": f"replicas x{world}" if world > 1 else "single"}


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
# algorithmic bytes of one substep (D bytes per real: 8 at FP64): particles 81 D N, pairs 16 P,
# contacts 2 C (8 + 16 D), manifolds M (12 + 20 D), colouring 12 (M + C), ledger M (16 + 8 D),
# velocity sweeps I_v M (12 + 20 D + 53 D), stabilization sweeps I_s M (the same per sweep),
# position sweeps I_p C (8 + 48 D)
def substep_bytes(n, P, C, M, iv, ip, D=8, istab=0.0):
    Sm = 12 + 20 * D
    return (81 * D * n + 16 * P + 2 * C * (8 + 16 * D) + M * Sm + 12 * (M + C) + M * (16 + 8 * D)
            + (iv + istab) * M * (Sm + 53 * D) + ip * C * (8 + 48 * D))


def stage_bytes(n, P, C, M, iv, istab, ip, D=8):
    """Algorithmic bytes of one substep per stage (the terms of substep_bytes)."""
    Sm = 12 + 20 * D
    return {"velocity": iv * M * (Sm + 53 * D), "stabilization": istab * M * (Sm + 53 * D),
            "position": ip * C * (8 + 48 * D), "broadphase": n * 4 * D + 8 * P,
            "narrowphase": 8 * P + C * (8 + 16 * D), "manifolds": 2 * C * (8 + 16 * D) + M * Sm,
            "colour_velocity": 12 * (M + C), "ledger": M * (16 + 8 * D)}


# DRAM traffic per substep of a stage from one ncu capture of the same workload (bytes per
# substep; stages not captured report none): the stabilization sweep loop of the 4,096-sphere
# restart (kSweepLoop<double, 3, 2, true>, one launch a substep: 3.23 MB read + 0.03 MB written;
# the state is L2-resident, so DRAM sees little of the loop's 148 MB of algorithmic traffic)
STAGE_DRAM_BYTES = {("plain_settling_4096_fp64", "stabilization"): 3.257e6}


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


def rank_range(n_items, rank, world):
    """Contiguous share [lo, hi) of n_items for rank (the calibration scenes)."""
    return (n_items * rank) // world, (n_items * (rank + 1)) // world


class L2Flush:
    """Writes a buffer larger than L2 (126 MB) on the current stream and waits for it."""

    def __init__(self):
        import torch
        self.torch = torch
        self.buf = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def __call__(self):
        self.buf.fill_(1.0)
        self.torch.cuda.synchronize()


# ---------------------------------------------------------------------------------------------
# headline: the plain XPBD settling configuration from its saved state
def outer_step(sim, sc):
    for _ in range(sc.substeps):
        sim.step(sc.dt)


def run_headline(args, rank, world, dist, dem, W):
    import torch
    sc = W.plain_settled()
    n = sc.n
    flush = L2Flush()

    def barrier():
        if dist is not None:
            dist.barrier()

    sim = sc.apply(dem.Simulation(n + 8, "fp64"))
    for _ in range(args.warmup):
        outer_step(sim, sc)
    sim.get_positions()  # synchronise
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    allocs = dem._API.fn["debug_allocs"]
    with clocks:
        time.sleep(0.5)  # sampler running before the timed region starts
        barrier()
        a0 = allocs()
        dev_ms = 0.0
        t0 = time.perf_counter()
        for _ in range(args.steps):
            flush()
            sim.timer_start()  # events on the library's stream around each timed outer step
            outer_step(sim, sc)
            dev_ms += sim.timer_stop()
        wall = time.perf_counter() - t0
        timed_allocs = allocs() - a0
    barrier()
    t_max = max_over_ranks(dev_ms / 1e3, dist, "cuda")
    value = aggregate_rate(world, n, SUBSTEPS, args.steps, t_max)
    # the same number of steps again with per-stage events (their synchronisation slows the step;
    # these explain the timed value, they are not it)
    sim.profile_enable(True)
    for _ in range(args.steps):
        outer_step(sim, sc)
    stages, launches = sim.profile_read()
    sweeps = sim.debug_sweeps()
    counts = sim.debug_counts()
    last = sim.counters()
    sim.profile_enable(False)
    x_end = sim.get_positions()
    v_end = sim.get_velocities()
    w_end = sim.get_angular_velocities()
    sim.close()

    # ---- the float step and the FP32-mixed form on the same window, and their distance from the
    # FP64 run after the same outer steps (warm-up, timed, and the profiled ones) ----
    other = {}
    for prec in ("fp32", "mixed"):
        sim = sc.apply(dem.Simulation(n + 8, prec))
        for _ in range(args.warmup):
            outer_step(sim, sc)
        sim.get_positions()
        ms = 0.0
        for _ in range(args.steps):
            flush()
            sim.timer_start()
            outer_step(sim, sc)
            ms += sim.timer_stop()
        for _ in range(args.steps):
            outer_step(sim, sc)
        err = np.linalg.norm(sim.get_positions() - x_end, axis=1) / sc.global_scale
        sim.close()
        t = max_over_ranks(ms / 1e3, dist, "cuda")
        other[prec] = {"value": aggregate_rate(world, n, SUBSTEPS, args.steps, t),
                       "max_position_error_radii": max_over_ranks(float(err.max()), dist, "cuda"),
                       "median_position_error_radii": float(np.median(err)),
                       "after_outer_steps": args.warmup + 2 * args.steps}

    # ---- end to end through the public API with host buffers, from the same state ----
    pinned = lambda: torch.zeros((n, 3), dtype=torch.float64, pin_memory=True).numpy()
    force, pos, vel = pinned(), pinned(), pinned()
    sim = sc.apply(dem.Simulation(n + 8, "fp64"))
    for _ in range(args.warmup):
        outer_step(sim, sc)
    sim.get_positions()
    barrier()
    a1 = allocs()
    laps = []
    for _ in range(args.steps):
        flush()
        tl = time.perf_counter()
        sim.set_external_forces(force)
        outer_step(sim, sc)
        sim.get_positions(out=pos)
        sim.get_velocities(out=vel)
        laps.append(time.perf_counter() - tl)
    e2e_allocs = allocs() - a1
    sim.close()
    assert np.all(np.isfinite(pos)) and np.all(np.isfinite(vel))
    e2e_t = max_over_ranks(sum(laps), dist, "cuda")
    e2e = {"value": aggregate_rate(world, n, SUBSTEPS, args.steps, e2e_t), "unit": METRIC,
           "h2d_bytes_per_step": int(force.nbytes), "d2h_bytes_per_step": int(pos.nbytes + vel.nbytes),
           "ms_per_step_median": round(1e3 * statistics.median(laps), 3), "device_allocations": int(e2e_allocs)}

    # ---- roofline of the dominant stage (per substep: one launch of the sweep loop) ----
    subs = args.steps * SUBSTEPS
    per_sub = {k: ms / subs for k, (ms, c) in stages.items() if c}
    P, C, M = counts["pairs"], counts["contacts"], counts["manifolds"]
    iv, istab, ip = sweeps["velocity"] / subs, sweeps["stabilization"] / subs, sweeps["position"] / subs
    sb = stage_bytes(n, P, C, M, iv, istab, ip)
    peak, peak_kind = measured_peaks()
    roof_stage = max((k for k in per_sub if k in sb), key=lambda k: per_sub[k])
    st_ms = per_sub[roof_stage]
    achieved = sb[roof_stage] / (st_ms / 1e3) / 1e9 if st_ms > 0 else 0.0
    step_bytes = substep_bytes(n, P, C, M, iv, ip, istab=istab)
    roofline = {"bound": "hbm", "kernel": f"{roof_stage} stage, per substep", "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": STAGE_DRAM_BYTES.get(("plain_settling_4096_fp64", roof_stage)),
                "algorithmic_bytes": sb[roof_stage], "stage_ms": st_ms,
                "l2_resident": "working set ~4 MB in the 126 MB L2: latency-bound (sweep loop barriers and "
                               "dependent loads), the HBM fraction is context",
                "step_algorithmic_GBps": step_bytes * subs / (dev_ms / 1e3) / 1e9}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        lib, march = ref_omp_lib()
        if lib:
            threads = os.cpu_count() or 1
            v, el, _ = cpu_reference_steps(sc, lib, threads, 3, args.cpu_steps)
            cpu = {"value": v, "unit": METRIC, "cores": threads, "kind": "reference",
                   "sample": f"{args.cpu_steps}x10 substeps of the restart after 3 warm-up, {el:.1f} s; "
                             f"reference on the OpenMP shim, float, -march={march}"}
    from peclet.dem import stats as S
    pk = S.packing_stats(x_end, np.full(n, sc.global_scale), 1.0 / sc.inv_mass, v_end, w_end,
                         1.0 / sc.inv_inertia[:, 0], sc.domain[0], sc.domain[1])
    return {"value": value, "t_max": t_max, "dev_ms": dev_ms, "wall": wall, "e2e": e2e, "roofline": roofline,
            "cpu": cpu, "clocks": clocks.summary(), "launches": launches, "timed_allocs": int(timed_allocs),
            "stages_ms_per_substep": {k: round(v, 4) for k, v in per_sub.items()},
            "sweeps_per_substep": {"velocity": iv, "stabilization": istab, "position": ip},
            "counts_last_substep": {"pairs": P, "contacts": C, "manifolds": M,
                                    "colours": [last["colors_velocity"], last["colors_position"]]},
            "packing_at_end": pk, "other_precisions": other}


# ---------------------------------------------------------------------------------------------
def cpu_reference_steps(scene, lib, threads, warm, steps):
    """The reference's own substep (a build under oracle/_ref) on `scene` for `warm` untimed and
    `steps` timed outer steps of scene.substeps calls; returns (particle-substeps/s, seconds,
    per-step seconds). The reference computes in float; the state is set as on the GPU."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    os.environ.setdefault("OMP_PROC_BIND", "close")
    capi = capi_module()
    sim = scene.apply(capi.CApiSimulation(capi.CApi(lib, "ref"), scene.n + 8, "fp32"))
    for _ in range(warm):
        outer_step(sim, scene)
    laps = []
    for _ in range(steps):
        t = time.perf_counter()
        outer_step(sim, scene)
        laps.append(time.perf_counter() - t)
    sim.close()
    el = sum(laps)
    return scene.n * scene.substeps * steps / el, el, laps


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    lib, march = ref_omp_lib()
    if lib is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/libref_omp*.so missing"}))
        return 0
    threads = os.cpu_count() or 1
    W = workloads_module()
    sc = W.plain_settled()
    value, el, laps = cpu_reference_steps(sc, lib, threads, args.warmup, args.steps)
    cfg = headline_desc(1)
    cfg["precision"] = "fp32 (the reference computes in float)"
    cfg["l2"] = "host run"
    cfg["parallelism"] = f"OpenMP, {threads} threads"
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded), saved restart state",
        "config": cfg, "impl": "reference",
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "reference",
                         "sample": f"{args.steps} outer steps (x10 substeps) of the 4096-sphere restart after "
                                   f"{args.warmup} warm-up steps; reference headers on the OpenMP Kokkos shim, "
                                   f"-O3 -march={march}, {threads} threads"},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
    return 0


# ---------------------------------------------------------------------------------------------
# extras
def run_xpbd262k(args, rank, world, dist, dem, W):
    """262,144 polydisperse spheres (lognormal radii, median 1 mm, sigma 0.25, clipped [0.5, 2] mm)
    placed by random sequential addition at solids fraction 0.35 in a box periodic in x and y with
    a floor, through the XPBD step (FP64, 10 substeps of 2e-6 s), timed after 100 untimed outer
    steps. This particle set is the Hertz configuration's; the reference names no XPBD
    configuration on it, so this line has no reference arm."""
    sc = W.polydisperse(n=262144)
    sim = sc.apply(dem.Simulation(sc.n + 8, "fp64"))
    for _ in range(100):
        outer_step(sim, sc)
    steps = args.extra_steps
    if dist is not None:
        dist.barrier()
    sim.timer_start()
    for _ in range(steps):
        outer_step(sim, sc)
    t = max_over_ranks(sim.timer_stop() / 1e3, dist, "cuda")
    c = sim.counters()
    sim.close()
    return {"workload": f"polydisperse_{sc.n}_periodic_xy_floor_xpbd_fp64", "value": aggregate_rate(world, sc.n, 10, steps, t),
            "ms_per_step": 1e3 * t / steps, "timed_steps_from": 100, "steps": steps,
            "last_substep": {k: c[k] for k in ("contacts", "manifolds", "velocity_sweeps", "position_sweeps")}}


def run_batched(args, rank, world, dist, dem, W):
    """Batched rotating drums (512 scenes) in one simulation per GPU, after their deposition: the
    drums are filled by random sequential addition in their lower halves and stepped
    `--drum-presettle` untimed outer steps in FP64 (the grains fall into a bed and the drums turn);
    that state is the start of an FP64 and an FP32-mixed run of the same warm-up and timed steps.
    The mixed form's error is its largest position difference from the FP64 run at the end, in
    radii. Scenes are split over the ranks with no exchange while stepping."""
    from peclet.dem.batch import apply_batch
    scenes, extras = W.rotating_drums(scenes=args.drums)
    mine = split_scenes([sc.n for sc in scenes], world)[rank]
    sc_m = [scenes[s] for s in mine]
    n_all = sum(sc.n for sc in scenes)
    n_mine = sum(sc.n for sc in sc_m)
    radius = np.concatenate([sc.scales * sc.global_scale for sc in sc_m])
    dt = sc_m[0].dt
    # deposition: one FP64 run from the RSA fill; its end state starts both timed runs
    for sc in sc_m:  # deposition: the grains start falling at 0.5 m/s (gravity is -y)
        sc.vel = sc.vel + np.array([0.0, -0.5, 0.0])
    sim = dem.Simulation(n_mine + 8, "fp64")
    first = apply_batch(sim, sc_m, [extras[s] for s in mine])
    for _ in range(args.drum_presettle * SUBSTEPS):
        sim.step(dt)
    x0, v0, q0, w0 = sim.get_positions(), sim.get_velocities(), sim.get_quaternions(), sim.get_angular_velocities()
    sim.close()
    t_dep = args.drum_presettle * SUBSTEPS * dt
    for k, s in enumerate(mine):  # restart each scene from its deposited state, walls turned on
        sl = slice(int(first[k]), int(first[k + 1]))
        sc_m[k].pos, sc_m[k].vel, sc_m[k].quat, sc_m[k].angvel = x0[sl], v0[sl], q0[sl], w0[sl]

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
        tune = {"sweep_loops": sim.scene_block(), "colouring": sim.color_block()}
        x = sim.get_positions()
        sim.close()
        return t, sweeps, x, tune

    t64, sw64, x64, tu64 = one("fp64")
    tmx, swmx, xmx, tumx = one("mixed")
    err = np.linalg.norm(xmx - x64, axis=1) / radius
    err_max = max_over_ranks(float(err.max()) if err.size else 0.0, dist, "cuda")
    rate = lambda t: n_all * SUBSTEPS * args.steps / t
    return {"workload": f"rotating_drums_{len(scenes)}_scenes_after_deposition", "scenes": len(scenes),
            "particles": n_all, "deposition_s": t_dep, "presettle_steps": args.drum_presettle,
            "fp64": {"value": rate(t64), "ms_per_step": 1e3 * t64 / args.steps, "autotuned_launch_shapes": tu64,
                     "mean_sweeps_last_substep": {"velocity": float(sw64[:, 2].mean()),
                                                  "stabilization": float(sw64[:, 3].mean()),
                                                  "position": float(sw64[:, 4].mean())}},
            "mixed": {"value": rate(tmx), "ms_per_step": 1e3 * tmx / args.steps, "autotuned_launch_shapes": tumx,
                      "err_vs_fp64": {"max_position_error_radii": err_max,
                                      "median_position_error_radii": float(np.median(err)) if err.size else 0.0,
                                      "after_substeps": (args.warmup + args.steps) * SUBSTEPS}},
            "mixed_over_fp64": t64 / tmx,
            "config": "R 50 mm, L 20 mm drums, omega U[0.5,3] rad/s, N_s U{256..8192} capped at 30% fill of the "
                      "lower half, radii U[0.8,1.2] mm, mu U[0.2,0.8], e U[0.3,0.9], dt 5e-5 s / 10 substeps"}


def run_calibration(args, rank, world, dist):
    """Differentiable calibration: boxes of 2048 spheres (r 1 mm, 40 x 40 x 80 mm, six planes),
    2000 Hertz substeps of 2e-5 s with checkpoints every 100, loss = mean squared distance of the
    final positions to targets made by the same solver at hidden (E, e, mu) = (5e6, 0.7, 0.35);
    gradients with respect to (E, e, mu) and the initial velocities from the adjoint, at the guess
    (4e6, 0.6, 0.3). Scenes are split over ranks; the three material gradients are summed over
    ranks with one all-reduce per backward pass. Reports forward-only and forward+adjoint rates
    (device time, max over ranks), their cost ratio, and the gradients' relative error against
    central finite differences (relative step 1e-4, FP64) on the 64-substep horizon, whose active
    contact set the check certifies unchanged at +h and -h, and on the full horizon (where contacts
    begin and end: a stated limitation), against the tangent-linear run, and FP32 against FP64."""
    import torch
    from peclet.dem import workloads as W
    from peclet.dem.adjoint import HertzSpheres
    per = 2048
    c = W.calibration_boxes(scenes=args.calib_scenes)
    lo, hi = rank_range(args.calib_scenes, rank, world)
    sl = slice(lo * per, hi * per)
    n_all = args.calib_scenes * per
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
    (xt, _, _), _ = s64.run(x0, v0, w0, hidden, steps)

    def ranks_sum(x):
        if dist is None:
            return float(x)
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        dist.all_reduce(t)
        return float(t)

    def loss_of(sim, theta, target, nsteps, vv=None):
        (x, _, _), _ = sim.run(x0, v0 if vv is None else vv, w0, tuple(theta), nsteps)
        return ranks_sum(((x.double() - target) ** 2).sum()) / n_all

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

    rel = lambda a, b: abs(a - b) / abs(b) if b else None
    gen = torch.Generator(device="cpu").manual_seed(5)
    dv = torch.randn(v0.shape, generator=gen, dtype=torch.float64).to(dev)
    dth = np.array([1e5, 0.01, 0.01])

    def all_ranks(flag):
        if dist is None:
            return bool(flag)
        t = torch.tensor([0.0 if flag else 1.0], dtype=torch.float64, device=dev)
        dist.all_reduce(t)
        return float(t) == 0.0

    def checks(nsteps, target, g64, gv64, g32, gv32, certify):
        """Central differences (relative step 1e-4) along E, e, mu and along a direction of the
        initial velocities of each rank's first scene; with `certify`, each difference is marked
        certified when the +h and -h rollouts touch exactly the contacts of the nominal one in
        every substep (no contact begins or ends between them: the rollout is smooth there)."""
        base = s64.active_sets(x0, v0, w0, guess, nsteps) if certify else None
        same = lambda vv, th: all_ranks(HertzSpheres.same_branches(s64.active_sets(x0, vv, w0, th, nsteps), base))
        fd, cert = [], []
        for k in range(3):
            h = 1e-4 * guess[k]
            tp, tm = list(guess), list(guess)
            tp[k] += h
            tm[k] -= h
            fd.append((loss_of(s64, tp, target, nsteps) - loss_of(s64, tm, target, nsteps)) / (2 * h))
            cert.append(same(v0, tp) and same(v0, tm) if certify else None)
        dv1 = dv.clone()
        dv1[per:] = 0.0  # the rank's first scene only
        hv = 1e-4 * 0.2
        fdv = (loss_of(s64, guess, target, nsteps, v0 + hv * dv1) - loss_of(s64, guess, target, nsteps, v0 - hv * dv1)) / (2 * hv)
        gotv = ranks_sum((gv64 * dv1).sum())
        certv = (same(v0 + hv * dv1, guess) and same(v0 - hv * dv1, guess)) if certify else None
        got = ranks_sum((gv64 * dv).sum()) + float((g64 * dth).sum())
        ((xj, _, _), (xdj, _, _)), _ = timed(lambda: s64.jvp(x0, v0, w0, guess, torch.zeros_like(x0), dv,
                                                            torch.zeros_like(w0), dth, nsteps))
        jv = ranks_sum((2.0 * (xj - target) * xdj).sum()) / n_all
        out = {"substeps": nsteps, "rel_err_vs_fd_1e-4": [rel(g64[k], fd[k]) for k in range(3)],
               "v0_first_scene_rel_err_vs_fd_1e-4": rel(gotv, fdv),
               "direction_rel_err_vs_tangent_linear": rel(got, jv),
               "fp32_rel_err_vs_fp64": [float(abs(a - b) / abs(b)) for a, b in zip(g32, g64)],
               "fp32_v0_rms_rel_err": float((gv32 - gv64).norm() / gv64.norm())}
        if certify:
            out["fd_certified"] = {"E": cert[0], "e": cert[1], "mu": cert[2], "v0_first_scene": certv}
            # the FP32 rollout's own branches against the FP64 one's: where they differ, the two
            # gradients are derivatives of different smooth pieces
            a32 = s32.active_sets(x0, v0, w0, guess, nsteps)
            out["fp32_substeps_with_other_branches"] = sum(
                int(not (p.numel() == q.numel() and bool(torch.equal(p, q)))) for p, q in zip(a32, base))
        return out

    out = {}
    grads = {}
    s32 = make("fp32")
    for prec, sim in (("fp64", s64), ("fp32", s32)):
        fwd_adj(sim, xt, min(steps, 2 * ck))  # warm-up: allocator, module loading, first launches
        _, t_f = timed(lambda: sim.run(x0, v0, w0, guess, steps))
        (g, gv), t_fa = timed(lambda: fwd_adj(sim, xt, steps))
        grads[prec] = (g, gv)
        out[prec] = {"forward": n_all * steps / t_f, "fwd_adjoint": n_all * steps / t_fa, "cost_ratio": t_fa / t_f}
    full = checks(steps, xt, *grads["fp64"], *grads["fp32"], certify=False)
    short = min(64, steps)
    (xs, _, _), _ = s64.run(x0, v0, w0, hidden, short)
    window = checks(short, xs, *fwd_adj(s64, xs, short), *fwd_adj(s32, xs, short), certify=True)
    return {"workload": f"calibration_boxes_{args.calib_scenes}x{per}", "particles": n_all, "substeps": steps,
            "checkpoint_every": ck, "path": "step_hertz force law (spheres, planes), hand-written adjoint",
            "fp64": out["fp64"], "fp32": out["fp32"], "checks_64_substeps": window, "checks_full_horizon": full,
            "full_horizon_note": "contacts begin and end inside 2000 substeps; central differences there do not "
                                 "converge as the step shrinks (kinks at contact onsets), the tangent-linear run "
                                 "is the check (a stated limitation, not certified)"}


def run_xpbd_adjoint(args, rank, world, dist, dem, W):
    """Adjoint of the XPBD substep on the headline scene (the 4,096-sphere bed of the plain settling
    configuration, FP64, from its saved restart): `--xadj-substeps` substeps recorded, then the
    backward of L = sum(a . x_end) + sum(b . v_end) with seeded weights. Reports the plain forward,
    the recording forward and the backward (device time on the library's stream, max over ranks;
    each rank runs its own replica) and the cost ratio (recording forward + backward) / plain
    forward; the finite-difference check runs on a calibration box (xpbd_fd_check). The
    dual-number check of the gradients, on this bed too, runs in the GPU tests."""
    import ctypes
    import torch
    from peclet.dem.xpbd_adjoint import XpbdRollout
    sc = W.plain_settled()
    T = args.xadj_substeps
    sim = sc.apply(dem.Simulation(sc.n + 8, "fp64"))
    roll = XpbdRollout(sim)
    dev = torch.device("cuda", torch.cuda.current_device())
    q0 = sc.quat if sc.quat is not None else np.tile([0.0, 0.0, 0.0, 1.0], (sc.n, 1))
    w0 = sc.angvel if sc.angvel is not None else np.zeros((sc.n, 3))
    start = [torch.tensor(np.asarray(a, np.float64), device=dev) for a in (sc.pos, q0, sc.vel, w0)]
    theta0 = np.array(sc.material, np.float64)
    rng = np.random.default_rng(7)
    A = torch.tensor(rng.normal(size=(sc.n, 3)), device=dev)
    Bv = torch.tensor(rng.normal(size=(sc.n, 3)) * 1e-3, device=dev)
    f, h = sim._f, sim._h
    P = lambda t: ctypes.c_void_p(t.data_ptr())

    def begin(th, v=None):
        sim.set_material_params(*[float(x) for x in th])
        rows = [start[0], start[1], start[2] if v is None else v, start[3]]
        torch.cuda.synchronize()
        roll._check(f["xa_begin"](h, *[P(t) for t in rows], sc.n), "xa_begin")

    def timed(fn):
        sim.timer_start()
        fn()
        return max_over_ranks(sim.timer_stop() / 1e3, dist, "cuda")  # ms -> s

    # warm-up, then the plain forward, the recording forward and the backward
    begin(theta0)
    roll._check(f["xa_step"](h, sc.dt, min(T, 10)), "xa_step")
    begin(theta0)
    t_plain = timed(lambda: [sim.step(sc.dt) for _ in range(T)])
    begin(theta0)
    t_rec = timed(lambda: roll._check(f["xa_step"](h, sc.dt, T), "xa_step"))
    sig0 = roll.signature()
    z = {c: torch.zeros((sc.n, c), dtype=torch.float64, device=dev) for c in (3, 4)}
    d = [torch.empty((sc.n, c), dtype=torch.float64, device=dev) for c in (3, 4, 3, 3)]
    dth = (ctypes.c_double * 3)()
    torch.cuda.synchronize()
    t_bwd = timed(lambda: roll._check(f["xa_backward"](h, P(A), P(z[4]), P(Bv), P(z[3]), *[P(t) for t in d], dth),
                                      "xa_backward"))
    info = roll.info()
    fd_check = xpbd_fd_check(args, dem, W)
    rate = lambda t: sc.n * T / t
    return {"workload": f"plain_settling_4096 restart (step {W.PLAIN_SETTLED_STEPS}), {T} substeps",
            "path": "plain FP64 XPBD step (coloured PGS, one-sided stabilization, position GS), recorded; "
                    "hand-written reversal over the frozen colouring",
            "forward_plain": rate(t_plain), "forward_recording": rate(t_rec), "fwd_adjoint": rate(t_rec + t_bwd),
            "cost_ratio": (t_rec + t_bwd) / t_plain, "backward_ms_per_substep": 1e3 * t_bwd / T,
            "forward_ms_per_substep": 1e3 * t_plain / T, "record_mb": info["record_bytes"] / 1e6,
            "work_mb": info["work_bytes"] / 1e6, "replay_dx_scale_units": info["replay_dx"],
            "fd_check": fd_check, "mean_sweeps": {k: float(v) for k, v in zip(
                ("velocity", "stabilization", "position"), sig0[:, 4:7].mean(axis=0))}}


def xpbd_fd_check(args, dem, W):
    """Central differences (relative step 1e-5, FP64) of L = sum(a . x_end) + sum(b . v_end) along
    eN, mu and a direction of the start velocities, against the adjoint, on the first box of the
    calibration workload (2048 spheres, the plain XPBD step at dt 2e-5) after `--xadj-fd-presettle`
    substeps (the collisional regime, about 200 contacts). A difference is certified when the +h
    and -h rollouts took the nominal one's discrete decisions (record signature) and branches
    (branch hash): the longest of the windows 16, 8, 4, 2 substeps that certifies all three is
    reported (a contact onset, a flipped clamp or adaptive stop is a jump the derivative does not
    see). On a settled bed no window certifies: contacts sit at the restitution cut-off and the
    impulse clamps, and any perturbation flips some; the dual-number check of the tests covers it."""
    import ctypes
    import torch
    from peclet.dem.xpbd_adjoint import XpbdRollout
    sc = W.calibration_box_scene(0)
    sim = sc.apply(dem.Simulation(sc.n + 8, "fp64"))
    for _ in range(args.xadj_fd_presettle):
        sim.step(sc.dt)
    roll = XpbdRollout(sim)
    dev = torch.device("cuda", torch.cuda.current_device())
    state = (sim.get_positions(), sim.get_quaternions(), sim.get_velocities(), sim.get_angular_velocities())
    start = [torch.tensor(np.asarray(a, np.float64), device=dev) for a in state]
    th0 = np.array(sc.material, np.float64)
    rng = np.random.default_rng(7)
    A = torch.tensor(rng.normal(size=(sc.n, 3)), device=dev)
    Bv = torch.tensor(rng.normal(size=(sc.n, 3)) * 1e-3, device=dev)
    dv = torch.tensor(np.random.default_rng(8).normal(size=(sc.n, 3)), device=dev)
    f, h = sim._f, sim._h
    P = lambda t: ctypes.c_void_p(t.data_ptr())

    def run(th, nsub, v=None):
        sim.set_material_params(*[float(x) for x in th])
        rows = [start[0], start[1], start[2] if v is None else v, start[3]]
        torch.cuda.synchronize()
        roll._check(f["xa_begin"](h, *[P(t) for t in rows], sc.n), "xa_begin")
        roll._check(f["xa_step"](h, sc.dt, nsub), "xa_step")
        x, v1 = sim.get_positions(), sim.get_velocities()
        L = float((A.cpu().numpy() * x).sum() + (Bv.cpu().numpy() * v1).sum())
        return L, (roll.signature(), roll.branches())

    same = lambda a, b: bool(np.array_equal(a[0], b[0]) and a[1] == b[1])
    rel = lambda a, b: abs(a - b) / abs(b) if b else None
    tried = []
    for win in (16, 8, 4, 2):
        _, sig = run(th0, win)
        d = [torch.empty((sc.n, c), dtype=torch.float64, device=dev) for c in (3, 4, 3, 3)]
        z = {c: torch.zeros((sc.n, c), dtype=torch.float64, device=dev) for c in (3, 4)}
        dth = (ctypes.c_double * 3)()
        torch.cuda.synchronize()
        roll._check(f["xa_backward"](h, P(A), P(z[4]), P(Bv), P(z[3]), *[P(t) for t in d], dth), "xa_backward")
        grads = {"eN": dth[0], "mu": dth[2], "v0": float((d[2] * dv).sum())}
        fd, cert = {}, {}
        for name, k in (("eN", 0), ("mu", 2)):
            hh = 1e-5 * th0[k]
            tp, tm = th0.copy(), th0.copy()
            tp[k] += hh
            tm[k] -= hh
            (lp, sp), (lm, sm) = run(tp, win), run(tm, win)
            fd[name] = (lp - lm) / (2 * hh)
            cert[name] = same(sp, sig) and same(sm, sig)
        hv = 1e-5 * 0.2
        (lp, sp), (lm, sm) = run(th0, win, start[2] + hv * dv), run(th0, win, start[2] - hv * dv)
        fd["v0"] = (lp - lm) / (2 * hv)
        cert["v0"] = same(sp, sig) and same(sm, sig)
        out = {"window_substeps": win, "grad": grads, "fd_1e-5": fd,
               "rel_err_vs_fd": {k: rel(grads[k], fd[k]) for k in fd}, "certified": cert}
        tried.append(win)
        if all(cert.values()):
            break
    out["workload"] = (f"calibration box 0 (2048 spheres, plain XPBD, dt 2e-5, (eN, eT, mu) = (0.6, 0, 0.3)) after "
                       f"{args.xadj_fd_presettle} substeps")
    out["windows_tried"] = tried
    return out


def run_hertz(args, rank, world, dist, dem, W):
    """The Hertz engine on the polydisperse packing (262,144 spheres), closed variant (the
    reference's engine refuses periodic domains and planes: floor and sides are one SDF grid
    wall), FP64 and FP32, after 20 untimed calls; the reference's own OpenMP build on the same
    scene beside it (a bounded sample of calls)."""
    sc, extra = W.polydisperse_hertz_closed()
    line = {"workload": f"polydisperse_{sc.n}_closed_hertz", "substeps_per_call": sc.substeps}
    for prec in ("fp64", "fp32"):
        sim = sc.apply(dem.Simulation(sc.n + 8, prec))
        extra(sim)
        for _ in range(20):
            sim.step_hertz(sc.dt, sc.substeps, 0.3)
        steps = args.extra_steps
        sim.timer_start()
        for _ in range(steps):
            sim.step_hertz(sc.dt, sc.substeps, 0.3)
        t = max_over_ranks(sim.timer_stop() / 1e3, dist, "cuda")
        line[prec] = {"value": aggregate_rate(world, sc.n, sc.substeps, steps, t), "ms_per_call": 1e3 * t / steps,
                      "calls_timed": steps, "timed_from_call": 20}
        sim.close()
    lib, march = ref_omp_lib()
    if rank == 0 and world == 1 and lib and not args.no_cpu:
        os.environ["OMP_NUM_THREADS"] = str(os.cpu_count() or 1)
        capi = capi_module()
        sim = sc.apply(capi.CApiSimulation(capi.CApi(lib, "ref"), sc.n + 8, "fp32"))
        extra(sim)
        sim.step_hertz(sc.dt, sc.substeps, 0.3)
        t = time.perf_counter()
        calls = 2
        for _ in range(calls):
            sim.step_hertz(sc.dt, sc.substeps, 0.3)
        el = time.perf_counter() - t
        sim.close()
        line["cpu_reference"] = {"value": sc.n * sc.substeps * calls / el, "cores": os.cpu_count(),
                                 "sample": f"{calls} calls after 1, {el:.1f} s, -march={march}"}
    return line


def run_shells(args, rank, world, dist, dem, W):
    """65,536 hollow cylinders (r_out 1 mm, r_in 0.6 mm, L 3 mm) with a seeded 512-point stratified
    shell. The configuration's 60 x 60 x 120 mm box cannot hold them (their solid volume is 91 % of
    it), so their bounding spheres are placed by random sequential addition at 25 % of a 1 x 1 x 2
    box (workloads.hollow_cylinders) and the line times the first outer steps from there, in FP64
    and the FP32-mixed form, with the mixed form's error against FP64 at the end. `--shell-presettle`
    steps of a gravity deposition (2 m/s downwards, substeps of four times the configuration's) run
    first when given; a dense shell bed is slow to build and to step (each touching pair carries up
    to 512 contacts), so the default is none."""
    sc = W.hollow_cylinders(shell_points=W.hollow_cylinder_shell())
    if args.shell_presettle > 0:
        sc = W.deposit(sc, dem, outer_steps=args.shell_presettle, v_down=2.0, dt_scale=4.0)
    line = {"workload": f"hollow_cylinders_{sc.n}_shell512" + ("_deposited" if args.shell_presettle else ""),
            "box_m": [float(v) for v in sc.domain[1]],
            "presettle_steps": args.shell_presettle}
    for prec in ("fp64", "mixed"):
        sim = sc.apply(dem.Simulation(sc.n + 8, prec))
        for _ in range(2):
            outer_step(sim, sc)
        steps = args.extra_steps
        sim.timer_start()
        for _ in range(steps):
            outer_step(sim, sc)
        t = max_over_ranks(sim.timer_stop() / 1e3, dist, "cuda")
        c = sim.counters()
        line[prec] = {"value": aggregate_rate(world, sc.n, sc.substeps, steps, t), "ms_per_step": 1e3 * t / steps,
                      "contacts_last_substep": c["contacts"], "position_sweeps_last_substep": c["position_sweeps"],
                      "velocity_sweeps_last_substep": c["velocity_sweeps"]}
        if prec == "fp64":
            x64 = sim.get_positions()
        else:
            err = np.linalg.norm(sim.get_positions() - x64, axis=1) / sc.global_scale
            line[prec]["err_vs_fp64"] = {"max_position_error_radii": float(err.max()),
                                         "after_substeps": (steps + 2) * sc.substeps}
        sim.close()
    return line


# ---------------------------------------------------------------------------------------------
def run_ours(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import peclet.dem as dem
    from peclet.dem import workloads as W
    dem._API.check(dem._API.fn["set_device"](local), "set_device")

    h = run_headline(args, rank, world, dist, dem, W)
    extras = [e for e in args.extras.split(",") if e in EXTRAS] if args.extras != "none" else []
    detail = {}
    runners = {"xpbd262k": lambda: run_xpbd262k(args, rank, world, dist, dem, W),
               "batched": lambda: run_batched(args, rank, world, dist, dem, W),
               "calibration": lambda: run_calibration(args, rank, world, dist),
               "xpbd_adjoint": lambda: run_xpbd_adjoint(args, rank, world, dist, dem, W),
               "hertz": lambda: run_hertz(args, rank, world, dist, dem, W),
               "shells": lambda: run_shells(args, rank, world, dist, dem, W)}
    for name in EXTRAS:
        if name in extras:
            detail[name] = runners[name]()

    if rank == 0:
        flat = {}
        if "xpbd262k" in detail:
            flat["xpbd262k_fp64_value"] = detail["xpbd262k"]["value"]
        if "batched" in detail:
            b = detail["batched"]
            flat.update(batched_fp64_value=b["fp64"]["value"], batched_mixed_value=b["mixed"]["value"],
                        batched_mixed_over_fp64=b["mixed_over_fp64"],
                        mixed_err_radii=b["mixed"]["err_vs_fp64"]["max_position_error_radii"])
        if "calibration" in detail:
            cb = detail["calibration"]
            c64 = cb["checks_64_substeps"]
            flat.update(fwd_adjoint_cost_ratio=cb["fp64"]["cost_ratio"], fwd_adjoint_value=cb["fp64"]["fwd_adjoint"],
                        grad_rel_err_vs_fd_64=max(v for v in c64["rel_err_vs_fd_1e-4"]
                                                  + [c64["v0_first_scene_rel_err_vs_fd_1e-4"]] if v is not None),
                        grad_fd_64_certified=all(c64["fd_certified"].values()),
                        grad_rel_err_vs_fd_full=max(v for v in cb["checks_full_horizon"]["rel_err_vs_fd_1e-4"]
                                                    if v is not None))
        if "xpbd_adjoint" in detail:
            xa = detail["xpbd_adjoint"]
            fc = xa["fd_check"]
            errs = [v for v in fc["rel_err_vs_fd"].values() if v is not None]
            flat.update(xpbd_fwd_adjoint_cost_ratio=xa["cost_ratio"], xpbd_fwd_adjoint_value=xa["fwd_adjoint"],
                        xpbd_grad_rel_err_vs_fd=max(errs) if errs else None,
                        xpbd_grad_fd_certified=all(fc["certified"].values()),
                        xpbd_grad_fd_window=fc["window_substeps"])
        if "hertz" in detail:
            flat.update(hertz262k_fp64_value=detail["hertz"]["fp64"]["value"],
                        hertz262k_fp32_value=detail["hertz"]["fp32"]["value"])
            if "cpu_reference" in detail["hertz"]:
                flat["hertz262k_cpu_reference_value"] = detail["hertz"]["cpu_reference"]["value"]
        if "shells" in detail:
            flat.update(shells_fp64_value=detail["shells"]["fp64"]["value"],
                        shells_mixed_value=detail["shells"]["mixed"]["value"])
        detail["headline"] = {k: h[k] for k in ("stages_ms_per_substep", "sweeps_per_substep", "counts_last_substep",
                                               "packing_at_end", "roofline", "other_precisions")}
        o = h["other_precisions"]
        flat.update(headline_fp32_value=o["fp32"]["value"], headline_mixed_value=o["mixed"]["value"],
                    headline_mixed_err_radii=o["mixed"]["max_position_error_radii"],
                    headline_fp32_err_radii=o["fp32"]["max_position_error_radii"])
        print(json.dumps({"detail": detail}))
        line = {
            "metric": METRIC, "value": h["value"], "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * h["t_max"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded), saved restart state",
            "config": headline_desc(world), "e2e": h["e2e"], "gpu_launches": h["launches"],
            "roofline": {k: h["roofline"][k] for k in ("bound", "kernel", "achieved", "peak", "unit", "frac",
                                                       "traffic", "peak_source")},
            "cpu_baseline": h["cpu"], "clocks": h["clocks"],
            "device_allocations_timed": h["timed_allocs"], **{k: _compact(v) for k, v in flat.items()}}
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


def _compact(v):
    """Six decimals for ordinary figures, three significant digits for small ones (errors)."""
    if not isinstance(v, float):
        return v
    return round(v, 6) if v == 0.0 or abs(v) >= 1e-3 else float(f"{v:.3g}")


def spawn_ranks(args):
    """`--gpus N` without a launcher: start N ranks on this node (one per GPU) through
    torch.distributed.run, which sets RANK / LOCAL_RANK / WORLD_SIZE, and pass their output on."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.run(cmd).returncode


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=20, help="timed outer steps of the headline's CPU baseline")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--extras", default=",".join(EXTRAS), help=f"comma list of {EXTRAS} or 'none'")
    ap.add_argument("--extra-steps", type=int, default=5, help="timed outer steps (or calls) of the extra lines")
    ap.add_argument("--drums", type=int, default=512)
    ap.add_argument("--drum-presettle", type=int, default=150, help="untimed FP64 outer steps of the drum deposition")
    ap.add_argument("--shell-presettle", type=int, default=0, help="untimed FP64 outer steps of a shell deposition")
    ap.add_argument("--calib-scenes", type=int, default=64)
    ap.add_argument("--calib-substeps", type=int, default=2000)
    ap.add_argument("--xadj-substeps", type=int, default=100, help="substeps of the XPBD adjoint line")
    ap.add_argument("--xadj-fd-presettle", type=int, default=200, help="substeps before its finite-difference check")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return spawn_ranks(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
