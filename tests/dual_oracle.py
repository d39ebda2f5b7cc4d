"""The FP64 oracle on forward-mode dual numbers (oracle/restate/orc_dual.hpp, precision 65).

`dual_sim` makes a `CApiSimulation` over the oracle's dual-number instantiation: the value run is
the FP64 oracle's, and `seed` / `tangent` set and read tangent lanes of the state (0 positions,
1 velocities, 2 angular velocities, 3 quaternions) or of the material (4: eN, eT, mu). With inputs
seeded, the tangents of the outputs are the directional derivatives of the plain FP64 solver along
the branch it took: the forward-mode check of the XPBD adjoint."""
import ctypes as C

import numpy as np

from peclet.dem._capi import CApiSimulation

POS, VEL, ANGVEL, QUAT, MATERIAL = 0, 1, 2, 3, 4
_COLS = {POS: 3, VEL: 3, ANGVEL: 3, QUAT: 4}


def dual_sim(orc_api, capacity):
    sim = CApiSimulation.__new__(CApiSimulation)
    sim._api, sim._f = orc_api, orc_api.fn
    sim.precision, sim._out_dtype = "fp64", np.float64
    h = C.c_void_p()
    orc_api.check(orc_api.fn["create"](int(capacity), 65, C.byref(h)), "dual oracle")
    sim._h = h
    return sim


def lanes(orc_api):
    return int(orc_api.lib.orc_dual_lanes())


def _fn(orc_api, name):
    f = getattr(orc_api.lib, name)
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double), C.c_long]
    return f


def seed(sim, which, lane, values):
    a = np.ascontiguousarray(np.asarray(values, np.float64).ravel())
    n = a.size if which == MATERIAL else a.size // _COLS[which]
    st = _fn(sim._api, "orc_dual_seed")(sim._h, which, lane, a.ctypes.data_as(C.POINTER(C.c_double)), n)
    sim._api.check(st, "orc_dual_seed")


def tangent(sim, which, lane, n):
    cols = 3 if which == MATERIAL else _COLS[which]
    size = 3 if which == MATERIAL else n * cols
    a = np.zeros(size, np.float64)
    st = _fn(sim._api, "orc_dual_get")(sim._h, which, lane, a.ctypes.data_as(C.POINTER(C.c_double)),
                                        3 if which == MATERIAL else n)
    sim._api.check(st, "orc_dual_get")
    return a if which == MATERIAL else a.reshape(n, cols)
