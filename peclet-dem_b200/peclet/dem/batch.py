"""Batched form: many independent scenes stepped together by one simulation.

The scenes' bodies are concatenated into one array; scene s owns bodies [first[s], first[s+1]).
Every launch of a substep covers all scenes, yet each scene is stepped exactly as a simulation of
that scene alone would step it (candidate pairs only inside a scene, its own contact margin,
restitution, friction, walls and adaptive iteration stops, and the colour priorities of its own
indices), so a batch reproduces the per-scene runs of the reference. Scenes may overlap in space.

Settings shared by the whole batch: shape, global scale, gravity, iterations, dt, e_t, planes and
the domain (the batch uses the first scene's; scenes with another domain change only the clamp
on oversized boxes). Per scene: bodies, restitution and friction (`Scene.material`), and the SDF
walls that its configuration callback adds.
"""
from __future__ import annotations

import numpy as np

from . import workloads as W


class _WallProxy:
    """What a scene's configuration callback sees: walls it adds belong to its scene."""

    def __init__(self, sim, scene):
        self._sim, self._scene, self._map = sim, scene, {}

    def add_sdf_wall(self, *args, **kw):
        wid = self._sim.add_sdf_wall(*args, **kw)
        self._sim.set_wall_scene(wid, self._scene)
        self._map[wid] = wid
        return wid

    def set_wall_velocity(self, wall_index, *args, **kw):
        self._sim.set_wall_velocity(wall_index, *args, **kw)

    def set_wall_material_id(self, wid, mat):
        self._sim.set_wall_material_id(wid, mat)


def concat(scenes):
    """One Scene holding every scene's bodies, and the scene table first[S+1]."""
    s0 = scenes[0]
    for sc in scenes[1:]:
        if (sc.shape != s0.shape or sc.global_scale != s0.global_scale or tuple(sc.gravity) != tuple(s0.gravity)
                or tuple(sc.iterations) != tuple(s0.iterations) or sc.dt != s0.dt or sc.material[1] != s0.material[1]
                or list(sc.planes) != list(s0.planes)):
            raise ValueError("batched scenes must share shape, scale, gravity, iterations, dt, e_t and planes")
        if (sc.quat is None) != (s0.quat is None) or (sc.shell is None) != (s0.shell is None):
            raise ValueError("batched scenes must all give (or all omit) orientations and shells")
    first = np.zeros(len(scenes) + 1, dtype=np.int64)
    first[1:] = np.cumsum([sc.n for sc in scenes])
    cat = lambda get: np.concatenate([get(sc) for sc in scenes], axis=0)
    scales = None
    if any(sc.scales is not None for sc in scenes):
        scales = cat(lambda sc: sc.scales if sc.scales is not None else np.ones(sc.n))
    big = W.Scene(name="batch", pos=cat(lambda sc: sc.pos), vel=cat(lambda sc: sc.vel),
                  inv_mass=cat(lambda sc: sc.inv_mass), inv_inertia=cat(lambda sc: sc.inv_inertia),
                  quat=cat(lambda sc: sc.quat) if s0.quat is not None else None, scales=scales,
                  shape=s0.shape, global_scale=s0.global_scale, domain=s0.domain, planes=list(s0.planes),
                  gravity=s0.gravity, material=s0.material, iterations=s0.iterations, dt=s0.dt,
                  substeps=s0.substeps, shell=s0.shell)
    return big, first


def apply_batch(sim, scenes, extras=None):
    """Configure `sim` (a Simulation with capacity >= the total body count) with the scenes.
    extras[s], when given, is the scene's configuration callback (walls, wall velocities)."""
    big, first = concat(scenes)
    big.apply(sim)
    sim.set_scenes(first)
    for s, sc in enumerate(scenes):
        sim.set_scene_material(s, sc.material[0], sc.material[2])
        if extras is not None and extras[s] is not None:
            extras[s](_WallProxy(sim, s))
    return first


class BatchSimulation:
    """A Simulation of several independent scenes (see the module docstring)."""

    def __init__(self, scenes, extras=None, precision="fp64", capacity=None):
        from . import Simulation
        total = int(sum(sc.n for sc in scenes))
        self.sim = Simulation(capacity or total + 8, precision)
        self.first = apply_batch(self.sim, scenes, extras)
        self.dt = scenes[0].dt

    def step(self, dt=None):
        self.sim.step(self.dt if dt is None else dt)

    def scene_slice(self, s):
        return slice(int(self.first[s]), int(self.first[s + 1]))

    def get_positions(self):
        return self.sim.get_positions()

    def get_velocities(self):
        return self.sim.get_velocities()

    def scene_counters(self):
        return self.sim.scene_counters()
