"""Packing statistics of a sphere bed: solids fraction, kinetic energy, coordination number.

Gauss-Seidel trajectories part ways chaotically, so two correct solvers agree on a settled bed
only statistically. These are the statistics the reference uses to judge a packing
(docs/packing_investigation.md:139-146: solids fraction, kinetic energy, and the coordination
number counted at a contact-gap tolerance of +0.002), computed from plain arrays so that the B200
step, the oracle and the reference build are measured by the same code.
"""
from __future__ import annotations

import numpy as np


def coordination(pos, radii, gap=0.002, mask=None):
    """Mean number of sphere neighbours within (r_i + r_j)(1 + gap) of each sphere in `mask`
    (all spheres when None), and the number of such spheres with no neighbour (rattlers)."""
    from scipy.spatial import cKDTree
    pos = np.asarray(pos, dtype=np.float64)
    radii = np.asarray(radii, dtype=np.float64)
    tree = cKDTree(pos)
    pairs = tree.query_pairs(2.0 * radii.max() * (1.0 + gap), output_type="ndarray")
    if pairs.size:
        d = np.linalg.norm(pos[pairs[:, 0]] - pos[pairs[:, 1]], axis=1)
        pairs = pairs[d < (radii[pairs[:, 0]] + radii[pairs[:, 1]]) * (1.0 + gap)]
    deg = np.bincount(pairs.ravel(), minlength=pos.shape[0]) if pairs.size else np.zeros(pos.shape[0], int)
    sel = deg if mask is None else deg[mask]
    return (float(sel.mean()) if sel.size else 0.0), int((sel == 0).sum())


def packing_stats(pos, radii, mass, vel, angvel, inertia, box_min, box_max, gap=0.002, skin=2.0):
    """Statistics of a bed settled on the floor of a closed box.

    - `phi`: solids fraction of the core of the bed: sphere centres inside the box shrunk by
      `skin` radii from the side walls and the floor, and below the bed height less `skin` radii
      (bed height: the 95th percentile of the centre heights); centre counting is unbiased away
      from the boundaries;
    - `ke`: total kinetic energy (translation plus rotation, scalar inertia), J;
    - `z`: mean coordination number of the core spheres at contact gap `gap` (relative to the
      sum of radii), `rattlers`: core spheres with no neighbour;
    - `bed_height`: the 95th percentile of the centre heights above the floor."""
    pos = np.asarray(pos, dtype=np.float64)
    radii = np.asarray(radii, dtype=np.float64)
    mass = np.broadcast_to(np.asarray(mass, dtype=np.float64), radii.shape)
    inertia = np.broadcast_to(np.asarray(inertia, dtype=np.float64), radii.shape)
    lo, hi = np.asarray(box_min, np.float64), np.asarray(box_max, np.float64)
    r = float(radii.max())
    top = float(np.percentile(pos[:, 2], 95.0))
    clo = lo + skin * r
    chi = np.array([hi[0] - skin * r, hi[1] - skin * r, top - skin * r])
    core = np.all((pos >= clo) & (pos <= chi), axis=1)
    vol = float(np.prod(np.maximum(chi - clo, 0.0)))
    phi = float((4.0 / 3.0 * np.pi * radii[core] ** 3).sum() / vol) if vol > 0 else 0.0
    ke = float(0.5 * (mass * (np.asarray(vel) ** 2).sum(1)).sum()
               + 0.5 * (inertia * (np.asarray(angvel) ** 2).sum(1)).sum())
    z, rattlers = coordination(pos, radii, gap, core)
    return {"phi": phi, "ke": ke, "z": z, "rattlers": rattlers, "core": int(core.sum()),
            "bed_height": top - float(lo[2])}
