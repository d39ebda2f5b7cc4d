"""peclet.dem on B200 — the XPBD substep of peclet-dem as hand-written sm_100a CUDA.

Drop-in for the reference's `peclet.dem` module (packaging/dem_init.py, src/dem_bindings.cpp):
`Simulation(capacity)` exposes the same methods, arguments and defaults, backed by the C ABI of
`libpdem.so` (include/pdem.h). `Simulation(capacity, precision="fp64")` (the default) runs the step
in double precision; `precision="fp32"` runs the reference's single-precision arithmetic.

The CUDA library is required: importing this package without `libpdem.so` raises ImportError, and
creating a Simulation without a CUDA device raises RuntimeError — there is no CPU fallback.
"""
from __future__ import annotations

import os

import numpy as np

from ._capi import CApi, CApiSimulation

__version__ = "0.3.2+b200"

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libpdem.so")
if not os.path.exists(_LIB_PATH):
    raise ImportError(
        f"peclet.dem: the CUDA library {_LIB_PATH} is missing; build it with "
        "`python peclet-dem_b200/build.py` (nvcc, sm_100a)")
_API = CApi(_LIB_PATH, "pdem")

execution_space = "CUDA sm_100a"


class Simulation(CApiSimulation):
    """The XPBD particle simulation (reference facade src/sim.hpp:909-1670) on one B200."""

    def __init__(self, capacity: int, precision: str = "fp64"):
        super().__init__(_API, capacity, precision)


def finalize():
    """Deterministic teardown hook of the reference module; device memory is owned per Simulation
    and released when it is closed or garbage-collected, so nothing is left to do here."""
    return None


def export_lammps(filename, step, pos, vel, quats, radii, box_min=None, box_max=None, pbc_enabled=False):
    """Module-level LAMMPS dump writer from raw arrays (src/dem_bindings.cpp:436-464, src/io.hpp:23-82)."""
    pos = np.asarray(pos, dtype=np.float32).reshape(-1, 3)
    vel = np.asarray(vel, dtype=np.float32).reshape(-1, 3)
    quats = np.asarray(quats, dtype=np.float32).reshape(-1, 4)
    radii = np.asarray(radii, dtype=np.float32).ravel()
    n = pos.shape[0]
    if box_min is not None and box_max is not None:
        lo, hi = np.asarray(box_min, np.float32), np.asarray(box_max, np.float32)
    elif n == 0:
        lo = hi = np.zeros(3, np.float32)
    else:
        lo = (pos - radii[:, None]).min(axis=0)
        hi = (pos + radii[:, None]).max(axis=0)
        m = np.float32(0.05) * (hi - lo)
        lo, hi = lo - m, hi + m
    with open(filename, "w") as f:
        f.write(f"ITEM: TIMESTEP\n{step}\nITEM: NUMBER OF ATOMS\n{n}\n")
        f.write(f"ITEM: BOX BOUNDS {'pp pp pp' if pbc_enabled else 'ff ff ff'}\n")
        for a in range(3):
            f.write(f"{lo[a]:g} {hi[a]:g}\n")
        f.write("ITEM: ATOMS id type x y z radius vx vy vz qw qx qy qz\n")
        for i in range(n):
            q = quats[i]
            f.write(f"{i + 1} 1 {pos[i, 0]:.6f} {pos[i, 1]:.6f} {pos[i, 2]:.6f} {radii[i]:.6f} "
                    f"{vel[i, 0]:.6f} {vel[i, 1]:.6f} {vel[i, 2]:.6f} {q[3]:.6f} {q[0]:.6f} {q[1]:.6f} {q[2]:.6f}\n")


__all__ = ["Simulation", "execution_space", "finalize", "export_lammps"]
