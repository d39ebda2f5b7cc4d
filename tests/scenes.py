"""Small seeded scenes that drive every branch of the substep for the parity tests.

Each builder returns a `workloads.Scene` (positions, velocities, masses, shape, domain, planes and
material settings) plus optional extra configuration applied after the scene (walls, materials,
thermostat, growth). Sizes are chosen so the oracle finishes a few dozen substeps in well under a
second.
"""
from __future__ import annotations

import numpy as np

from peclet.dem import workloads as W


def _cluster(rng, n, box, radius):
    lo, hi = np.array(box[0]) + radius, np.array(box[1]) - radius
    return lo + rng.uniform(0, 1, (n, 3)) * (hi - lo)


def dense_spheres(seed=11, n=300, box=((0, 0, 0), (8e-3, 8e-3, 8e-3)), radius=1e-3, vmax=0.3,
                  e=0.5, mu=0.5, gravity=(0, 0, -9.81), iters=(10, 10), dt=1e-5):
    """Overlapping random spheres in a closed box: many contacts, deep overlaps, all planes."""
    rng = np.random.default_rng(seed)
    pos = _cluster(rng, n, box, radius)
    im, iI = W.sphere_props(radius, 2500.0)
    return W.Scene(name="dense_spheres", pos=pos, vel=rng.uniform(-vmax, vmax, (n, 3)),
                   inv_mass=np.full(n, im), inv_inertia=np.full((n, 3), iI),
                   global_scale=radius, domain=(box[0], box[1], (False, False, False)),
                   planes=W.box_planes(box[0], box[1]), gravity=gravity, material=(e, 0.0, mu),
                   iterations=iters, dt=dt)


def settled_column(seed=12, nx=5, ny=5, nz=12, iters=(10, 10)):
    """A lattice column dropped onto the floor: persistent contacts, warm start, stabilization."""
    sc = W.plain_settling(seed=seed, nx=nx, ny=ny, nz=nz, cells_z=nz + 2, spacing_r=1.98,
                          jitter_r=0.02, vmax=0.05, iterations=iters)
    sc.name = "settled_column"
    return sc


def reversed_column(seed=12, nx=3, ny=3, nz=24):
    """A tall lattice column numbered top to bottom: every support chain runs against the
    manifold order, so the serial support-level sweeps move one level a sweep and stop short of
    the fixed point (the exact-sweep path of the support levels)."""
    sc = settled_column(seed=seed, nx=nx, ny=ny, nz=nz)
    r = slice(None, None, -1)
    sc.pos, sc.vel = sc.pos[r].copy(), sc.vel[r].copy()
    sc.inv_mass, sc.inv_inertia = sc.inv_mass[r].copy(), sc.inv_inertia[r].copy()
    sc.name = "reversed_column"
    return sc


def polydisperse_periodic(seed=13, n=250, L=8e-3, H=6e-3, radius=1e-3):
    """Polydisperse spheres in a box periodic in x and y with a floor plane (ghost images)."""
    rng = np.random.default_rng(seed)
    r = np.clip(rng.lognormal(np.log(radius), 0.25, n), 0.5 * radius, 2 * radius)
    pos = np.stack([rng.uniform(0, L, n), rng.uniform(0, L, n), rng.uniform(r, H)], axis=1)
    m = 2500.0 * 4 / 3 * np.pi * r ** 3
    iI = 1.0 / (0.4 * m * r ** 2)
    return W.Scene(name="poly_periodic", pos=pos, vel=rng.uniform(-0.2, 0.2, (n, 3)),
                   inv_mass=1.0 / m, inv_inertia=np.repeat(iI[:, None], 3, 1), scales=r / radius,
                   global_scale=radius, domain=((0, 0, 0), (L, L, H), (True, True, False)),
                   planes=[(0, 0, 0, 0, 0, 1)], material=(0.6, 0.0, 0.4), dt=1e-5)


def cylinders(seed=14, n=24, L=8e-3, shape_type=W.HOLLOW_CYLINDER, shell=None):
    """A few hollow cylinders (or cubes) with random orientations: point-shell narrowphase."""
    rng = np.random.default_rng(seed)
    s = 1e-3
    pos = _cluster(rng, n, ((0, 0, 0), (L, L, L)), 1.6 * s)
    q = W.random_unit_quats(rng, n)
    m = 1200.0 * np.pi * (1.0 - 0.36) * 3.0 * s ** 3
    if shape_type == W.HOLLOW_CYLINDER:
        shape = (W.HOLLOW_CYLINDER, 1.0, 3.0, 0.4)
        iI = np.tile([12 / (m * (3 * 1.36 + 9) * s * s), 2 / (m * 1.36 * s * s),
                      12 / (m * (3 * 1.36 + 9) * s * s)], (n, 1))
    else:
        shape = (W.BOX, 1.0, 0.0, 0.0)
        iI = np.full((n, 3), 6.0 / (m * 4 * s * s))
    return W.Scene(name=f"shells_{shape_type}", pos=pos, vel=rng.uniform(-0.3, 0.3, (n, 3)),
                   inv_mass=np.full(n, 1.0 / m), inv_inertia=iI, quat=q, shape=shape,
                   global_scale=s, domain=((0, 0, 0), (L, L, L), (False, False, False)),
                   planes=W.box_planes((0, 0, 0), (L, L, L)), material=(0.4, 0.0, 0.3),
                   iterations=(20, 10), dt=6.25e-6, shell=shell)


def capsule_sdf(radius=0.6, half=0.6, h=0.1, pad=0.2, n_shell=240, seed=16):
    """A capsule (axis y, canonical units) as a grid-SDF particle shape: the exact distance to its
    core segment minus the radius, sampled on a grid, with a seeded point shell on its surface and
    the unit-mass inverse inertia of a solid capsule (cylinder plus two hemispheres)."""
    rng = np.random.default_rng(seed)
    ext = half + radius + pad
    n = int(round(2 * ext / h)) + 1
    ax = -ext + h * np.arange(n)
    Z, Y, X = np.meshgrid(ax, ax, ax, indexing="ij")
    grid = np.sqrt(X ** 2 + (np.abs(Y) - np.minimum(np.abs(Y), half)) ** 2 + Z ** 2) - radius
    # shell: the cylinder by area, then the two hemispheres
    a_cyl, a_cap = 2 * np.pi * radius * 2 * half, 4 * np.pi * radius ** 2
    n_cyl = int(round(n_shell * a_cyl / (a_cyl + a_cap)))
    th = rng.uniform(0, 2 * np.pi, n_cyl)
    cyl = np.stack([radius * np.cos(th), rng.uniform(-half, half, n_cyl), radius * np.sin(th)], 1)
    d = rng.normal(size=(n_shell - n_cyl, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    cap = radius * d + np.stack([np.zeros(len(d)), np.sign(d[:, 1]) * half, np.zeros(len(d))], 1)
    shell = np.concatenate([cyl, cap])
    mc, ms = np.pi * radius ** 2 * 2 * half, 4 / 3 * np.pi * radius ** 3
    m = mc + ms
    iyy = mc * radius ** 2 / 2 + ms * 2 * radius ** 2 / 5
    ixx = mc * (3 * radius ** 2 + (2 * half) ** 2) / 12 + ms * (2 * radius ** 2 / 5 + half ** 2 + 3 * half * radius / 4)
    inv_i = np.array([m / ixx, m / iyy, m / ixx])
    return (grid.ravel(), n, n, n, (-ext, -ext, -ext), (h, h, h), shell, inv_i, half + radius)


def sdf_capsules(seed=17, n=30, L=8e-3):
    """Capsules given as a grid-SDF shape (set_sdf_shape), random orientations, in a closed box."""
    rng = np.random.default_rng(seed)
    s = 1e-3
    pos = _cluster(rng, n, ((0, 0, 0), (L, L, L)), 1.2 * s)
    m = 1500.0 * (np.pi * 0.36 * 1.2 + 4 / 3 * np.pi * 0.216) * s ** 3
    sdf = capsule_sdf()
    iI = np.tile(np.asarray(sdf[7]) / (m * s * s), (n, 1))
    return W.Scene(name="sdf_capsules", pos=pos, vel=rng.uniform(-0.3, 0.3, (n, 3)),
                   inv_mass=np.full(n, 1.0 / m), inv_inertia=iI, quat=W.random_unit_quats(rng, n),
                   global_scale=s, domain=((0, 0, 0), (L, L, L), (False, False, False)),
                   planes=W.box_planes((0, 0, 0), (L, L, L)), material=(0.4, 0.0, 0.3),
                   iterations=(20, 10), dt=6.25e-6, sdf=sdf)


drum_wall_grid = W.drum_wall_grid


def spheres_in_drum(seed=15, n=120, R=6e-3, length=4e-3, omega=2.0, e=0.5, mu=0.4):
    rng = np.random.default_rng(seed)
    r = 0.5e-3
    ang = rng.uniform(0, 2 * np.pi, n)
    rad = np.sqrt(rng.uniform(0, 1, n)) * (R - 1.5 * r)
    pos = np.stack([rad * np.cos(ang), -np.abs(rad * np.sin(ang)), rng.uniform(1.5 * r, length - 1.5 * r, n)], 1)
    im, iI = W.sphere_props(r, 2500.0)
    sc = W.Scene(name="drum", pos=pos, vel=rng.uniform(-0.1, 0.1, (n, 3)), inv_mass=np.full(n, im),
                 inv_inertia=np.full((n, 3), iI), global_scale=r,
                 domain=((-R, -R, 0), (R, R, length), (False, False, False)),
                 gravity=(0, -9.81, 0), material=(e, 0.0, mu), dt=1e-5)
    grid, nx, ny, nz, origin, spacing = drum_wall_grid(R, length)

    def extra(sim):
        wid = sim.add_sdf_wall(grid, nx, ny, nz, origin, spacing, 0.5, 0.6)
        sim.set_wall_velocity(wid, (0, 0, 0), (0, 0, omega), (0, 0, 0))
    return sc, extra


def shells_at_floor(seed=18, L=40e-3):
    """Hollow-cylinder shells held just above and below the reach of a floor plane (the largest
    shell-point norm times the scale, plus the contact margin): bodies at heights stepping through
    that bound, one orientation putting a rim corner straight down and others random."""
    rng = np.random.default_rng(seed)
    s = 1e-3
    reach = np.sqrt(1.0 + 1.5 ** 2) * s  # farthest shell point of (r_out 1, length 3)
    dz = np.array([-5e-4, -2e-4, -5e-5, 0.0, 5e-5, 1.2e-4, 1.6e-4, 1.8e-4, 2.0e-4, 2.4e-4, 5e-4])
    a = -np.arctan(1.5)  # about x: the corner (0, 1.5, -1) straight down
    corner = np.array([np.sin(a / 2), 0.0, 0.0, np.cos(a / 2)])
    pos, quat = [], []
    for k, h in enumerate(dz):
        for j, q in enumerate((corner, W.random_unit_quats(rng, 1)[0])):
            pos.append([3e-3 + 5.5e-3 * (k % 5), 3e-3 + 5.5e-3 * (2 * (k // 5) + j), reach + h])
            quat.append(q)
    pos, quat = np.array(pos), np.array(quat)
    n = len(pos)
    m = 1200.0 * np.pi * (1.0 - 0.36) * 3.0 * s ** 3
    iI = np.tile([12 / (m * (3 * 1.36 + 9) * s * s), 2 / (m * 1.36 * s * s), 12 / (m * (3 * 1.36 + 9) * s * s)],
                 (n, 1))
    return W.Scene(name="shells_at_floor", pos=pos, vel=np.zeros((n, 3)), inv_mass=np.full(n, 1.0 / m),
                   inv_inertia=iI, quat=quat, shape=(W.HOLLOW_CYLINDER, 1.0, 3.0, 0.4), global_scale=s,
                   domain=((0, 0, 0), (L, L, L), (False, False, False)), planes=W.box_planes((0, 0, 0), (L, L, L)),
                   material=(0.4, 0.0, 0.3), iterations=(20, 10), dt=6.25e-6)
