"""Seeded sphere scenes of the differentiable Hertz rollout (shared by its CPU and GPU tests).

A "gas" case is several scenes of a 3 x 3 x 3 lattice of r = 1 mm spheres with jitter in a closed
box (six planes) that the outer spheres nearly touch, random velocities and spins: sphere-sphere and sphere-plane collisions with
sliding and sticking friction inside a few dozen substeps. The smaller cases isolate one oblique
sphere pair and one sphere bouncing on a floor."""
from __future__ import annotations

import numpy as np

DENSITY = 2500.0
THETA = np.array([5e6, 0.7, 0.35])  # E [Pa], restitution, friction
NU = 0.3
DT = 2e-5


def props(r):
    r = np.asarray(r, np.float64)
    m = DENSITY * 4.0 / 3.0 * np.pi * r ** 3
    return m, 0.4 * m * r * r


def box(L):
    return [[0, 0, 0, 0, 0, 1], [0, 0, L, 0, 0, -1], [0, 0, 0, 1, 0, 0], [L, 0, 0, -1, 0, 0],
            [0, 0, 0, 0, 1, 0], [0, L, 0, 0, -1, 0]]


def gas(seed=3, scenes=2, gap=0.3e-3, vmax=0.2, spin=50.0, wall_gap=0.1e-3):
    """Lattice gaps `gap`, the outer spheres `wall_gap` from the box's planes.
    Returns dict(x0, v0, w0, r, m, I, first, planes, g)."""
    rng = np.random.default_rng(seed)
    o = 1e-3 + wall_gap
    L = 2 * o + 2 * (2e-3 + gap)
    xs = []
    for _ in range(scenes):
        g = np.stack(np.meshgrid(*[np.arange(3)] * 3, indexing="ij"), -1).reshape(-1, 3) * (2e-3 + gap) + o
        xs.append(g + rng.uniform(-0.04e-3, 0.04e-3, g.shape))
    x0 = np.concatenate(xs)
    n = len(x0)
    r = np.full(n, 1e-3)
    m, I = props(r)
    return dict(x0=x0, v0=rng.uniform(-vmax, vmax, (n, 3)), w0=rng.uniform(-spin, spin, (n, 3)), r=r, m=m, I=I,
                first=[27 * s for s in range(scenes + 1)], planes=box(L), g=(0.0, 0.0, -9.81))


def pair():
    x0 = np.array([[0, 0, 0], [1.99e-3, 0.1e-3, 0]])
    r = np.full(2, 1e-3)
    m, I = props(r)
    return dict(x0=x0, v0=np.array([[0.1, 0.05, 0], [-0.1, 0, 0.02]]), w0=np.array([[0, 0, 10.0], [5, 0, 0]]),
                r=r, m=m, I=I, first=[0, 2], planes=[], g=(0.0, 0.0, 0.0))


def floor():
    x0 = np.array([[0, 0, 0.99e-3]])
    r = np.full(1, 1e-3)
    m, I = props(r)
    return dict(x0=x0, v0=np.array([[0.1, 0.05, -0.1]]), w0=np.array([[1.0, 2, 3]]), r=r, m=m, I=I, first=[0, 1],
                planes=[[0, 0, 0, 0, 0, 1]], g=(0.0, 0.0, -9.81))


def shape_pairs(seed=31, n=40, L=8e-3, shell=None, calls_substeps=(4, 10)):
    """Hollow cylinders (point shells) under the Hertz engine: the shape-pair force path
    (src/solver_hertz.hpp:454, called at src/sim.hpp:696) and shell-wall contacts. The engine
    refuses analytic planes, so the container is one SDF grid wall (floor and sides of an open
    box). Returns (scene, extra)."""
    import scenes as S
    from peclet.dem import workloads as W
    sc = S.cylinders(seed=seed, n=n, L=L, shell=shell)
    sc.planes = []
    grid = W.box_wall_grid(L, L, h=0.5e-3)

    def extra(s):
        s.add_sdf_wall(*grid, 0.4, 0.3)
        s.set_hertz_material(0, 1e7, 0.3)
    return sc, extra
