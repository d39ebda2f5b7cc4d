"""Shared helpers of the parity tests: snapshots of a simulation's state and intermediate products,
and their comparison (exact for integers/indices, exact or relative tolerance for floating point)."""
import numpy as np

import scenes as S
from peclet.dem import workloads as W
from peclet.dem._capi import CApiSimulation

STATE_KEYS = ("pos", "vel", "quat", "angvel")
PRODUCT_KEYS = ("pairs", "contacts", "manifolds", "mcolor", "ccolor", "lambda", "pair_keys", "ledger_keys",
                "ledger", "grounded", "pos_lambda", "max_overlap")


def snapshot(sim, products=True):
    s = {"pos": sim.get_positions().astype(np.float64), "vel": sim.get_velocities().astype(np.float64),
         "quat": sim.get_quaternions().astype(np.float64),
         "angvel": sim.get_angular_velocities().astype(np.float64)}
    if products:
        k, led = sim.debug_ledger()
        s.update(pairs=sim.debug_pairs(), contacts=sim.debug_contacts(), manifolds=sim.debug_manifolds(),
                 mcolor=sim.debug_manifold_colors(), ccolor=sim.debug_contact_colors(), lambda_=None)
        s.pop("lambda_")
        s.update({"lambda": sim.debug_lambda(), "pair_keys": sim.debug_pair_keys(), "ledger_keys": k,
                  "ledger": led, "grounded": sim.debug_grounded(), "pos_lambda": sim.debug_pos_lambda(),
                  "max_overlap": np.array([sim.max_overlap()])})
    return s


def diff(a, b, rtol=0.0, keys=None):
    """Return a list of (key, message) mismatches between two snapshots."""
    bad = []
    for k in keys or a.keys():
        x, y = a[k], b[k]
        if x.shape != y.shape:
            bad.append((k, f"shape {x.shape} vs {y.shape}"))
            continue
        if x.dtype.kind in "iu" or rtol == 0.0:
            ok = np.array_equal(x, y, equal_nan=x.dtype.kind == "f")
            if not ok:
                idx = np.argwhere(~((x == y) | (np.isnan(x) & np.isnan(y)))) if x.dtype.kind == "f" else np.argwhere(x != y)
                first = tuple(idx[0])
                bad.append((k, f"{len(idx)} differ, first at {first}: {x[first]!r} vs {y[first]!r}"))
        else:
            scale = np.maximum(np.abs(y), np.finfo(np.float64).tiny)
            rel = np.abs(x - y) / scale
            absd = np.abs(x - y)
            # relative to the value, with an absolute floor at rtol times the array's magnitude
            floor = rtol * (np.max(np.abs(y)) if y.size else 0.0)
            bad_mask = (absd > rtol * np.abs(y)) & (absd > floor)
            if np.any(bad_mask):
                first = tuple(np.argwhere(bad_mask)[0])
                bad.append((k, f"{int(bad_mask.sum())} beyond rtol {rtol}, first {first}: {x[first]!r} vs {y[first]!r}"))
    return bad


def build(api, scene, extra=None, precision="fp32", capacity=None):
    sim = scene.apply(CApiSimulation(api, capacity or scene.n + 8, precision))
    if extra:
        extra(sim)
    return sim


def _mats(sim):
    ids = np.arange(sim.num_particles()) % 3
    sim.set_material_ids(ids)
    sim.set_pair_material(0, 1, 0.9, 0.1)
    sim.set_pair_material(2, 2, 0.2, 0.8)


def _drum():
    sc, ex = S.spheres_in_drum()
    return sc, ex


# (name, scene factory, extra configuration, substeps) — every branch of the substep
MATRIX = [
    ("dense_spheres", lambda: S.dense_spheres(), None, 12),
    ("g0_friction_onshot_gs", lambda: S.dense_spheres(gravity=(0, 0, 0)), None, 8),
    ("jacobi", lambda: S.dense_spheres(), lambda s: s.set_velocity_use_gs(False), 6),
    ("escalate", lambda: S.dense_spheres(), lambda s: s.set_stabilization_mode("escalate"), 6),
    ("stabilization_off", lambda: S.dense_spheres(), lambda s: s.set_stabilization_mode("off"), 6),
    ("settled_column", lambda: S.settled_column(), None, 25),
    ("periodic_polydisperse", lambda: S.polydisperse_periodic(), None, 10),
    ("hollow_cylinders", lambda: S.cylinders(), None, 6),
    ("boxes", lambda: S.cylinders(shape_type=W.BOX), None, 6),
    ("drum_sdf_wall", lambda: _drum()[0], lambda s: _drum()[1](s), 10),
    ("thermostat", lambda: S.dense_spheres(gravity=(0, 0, 0), mu=0.0), lambda s: s.set_thermostat(1e-9, 1e-3, 1.0), 5),
    ("growth", lambda: S.dense_spheres(gravity=(0, 0, 0), mu=0.0), lambda s: s.set_growth_params(50.0, 0.8), 5),
    ("pair_materials", lambda: S.dense_spheres(), _mats, 6),
    ("walton_beta", lambda: S.dense_spheres(), lambda s: s.set_material_params(0.5, 0.3, 0.5), 6),
    ("grid_sdf_capsules", lambda: S.sdf_capsules(), None, 8),
    ("reversed_column", lambda: S.reversed_column(), None, 40),
    ("ordered_column", lambda: S.settled_column(), lambda s: s.set_stabilization_mode("ordered"), 25),
    ("ordered_dense", lambda: S.dense_spheres(), lambda s: s.set_stabilization_mode("ordered"), 8),
    ("multilevel_column", lambda: S.settled_column(), lambda s: s.set_stabilization_mode("multilevel"), 25),
    ("multilevel_dense", lambda: S.dense_spheres(), lambda s: s.set_stabilization_mode("multilevel"), 10),
    ("multilevel_periodic", lambda: S.polydisperse_periodic(), lambda s: s.set_stabilization_mode("multilevel"), 10),
]
