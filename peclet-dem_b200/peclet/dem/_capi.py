"""ctypes binding of a `<prefix>_*` C ABI to the reference's `Simulation` method names.

The reference exposes `peclet.dem.Simulation` through nanobind (src/dem_bindings.cpp:72-432). This
module re-exposes the same methods (same names, argument meaning and defaults) over a plain C ABI
(`include/pdem.h`): every call is one `extern "C"` function taking host pointers and sizes, returning
an int status that is turned into the reference's exception types here (`std::invalid_argument` ->
ValueError, `std::runtime_error` -> RuntimeError, src/sim.hpp:1036-1042,1147-1149,1154-1155).

`CApiSimulation` is generic over the library and the symbol prefix so that every implementation of
the same ABI (the B200 library, and any checker built to the same ABI) is driven by one code path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_dbl_p = C.POINTER(C.c_double)
_int_p = C.POINTER(C.c_int)
_long_p = C.POINTER(C.c_long)
_u64_p = C.POINTER(C.c_ulonglong)
_vp = C.c_void_p

# precision code of the FP32-mixed form (include/pdem.h PDEM_MIXED)
PRECISION_MIXED = 3264

# status codes (include/pdem.h)
OK, ERR_RUNTIME, ERR_INVALID, ERR_UNSUPPORTED, ERR_CUDA = 0, 1, 2, 3, 4

# name -> (restype, argtypes) for the shared ABI (the prefix is prepended at load time)
_SIGS = {
    "last_error": (C.c_char_p, []),
    "set_device": (C.c_int, [C.c_int]),
    "create": (C.c_int, [C.c_int, C.c_int, C.POINTER(_vp)]),
    "destroy": (None, [_vp]),
    "initialize_shape": (C.c_int, [_vp, C.c_int, C.c_double, C.c_double, C.c_double]),
    "set_sdf_shape": (C.c_int, [_vp, _dbl_p, C.c_int, C.c_int, C.c_int, _dbl_p, _dbl_p, _dbl_p,
                                C.c_int, _dbl_p, C.c_double]),
    "set_shell_points": (C.c_int, [_vp, _dbl_p, C.c_int]),
    "set_domain": (C.c_int, [_vp, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int]),
    "set_domain_minmax": (C.c_int, [_vp, _dbl_p, _dbl_p]),
    "enable_periodicity": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int]),
    "set_gravity": (C.c_int, [_vp, C.c_double, C.c_double, C.c_double]),
    "set_thermostat": (C.c_int, [_vp, C.c_double, C.c_double, C.c_double]),
    "set_solver_iterations": (C.c_int, [_vp, C.c_int, C.c_int]),
    "set_velocity_use_gs": (C.c_int, [_vp, C.c_int]),
    "set_stabilization_mode": (C.c_int, [_vp, C.c_char_p]),
    "set_hertz_material": (C.c_int, [_vp, C.c_int, C.c_double, C.c_double]),
    "set_global_scale": (C.c_int, [_vp, C.c_double]),
    "set_dt": (C.c_int, [_vp, C.c_double]),
    "set_material_params": (C.c_int, [_vp, C.c_double, C.c_double, C.c_double]),
    "set_material_ids": (C.c_int, [_vp, _int_p, C.c_int]),
    "set_pair_material": (C.c_int, [_vp, C.c_int, C.c_int, C.c_double, C.c_double]),
    "set_wall_material_id": (C.c_int, [_vp, C.c_int, C.c_int]),
    "add_plane": (C.c_int, [_vp] + [C.c_double] * 6),
    "add_sdf_wall": (C.c_int, [_vp, _dbl_p, C.c_int, C.c_int, C.c_int, _dbl_p, _dbl_p, C.c_double,
                               C.c_double, _int_p]),
    "set_wall_velocity": (C.c_int, [_vp, C.c_int, _dbl_p, _dbl_p, _dbl_p]),
    "set_positions": (C.c_int, [_vp, _dbl_p, C.c_int]),
    "set_velocities": (C.c_int, [_vp, _dbl_p, C.c_int]),
    "set_external_forces": (C.c_int, [_vp, _dbl_p, C.c_int]),
    "clear_external_forces": (C.c_int, [_vp]),
    "set_quaternions": (C.c_int, [_vp, _dbl_p, C.c_int]),
    "set_angular_velocities": (C.c_int, [_vp, _dbl_p, C.c_int]),
    "set_inv_inertia": (C.c_int, [_vp, _dbl_p, C.c_int]),
    "set_inv_mass": (C.c_int, [_vp, _dbl_p, C.c_int]),
    "set_scales": (C.c_int, [_vp, _dbl_p, C.c_int]),
    "set_scales_uniform": (C.c_int, [_vp, C.c_double]),
    "set_growth_params": (C.c_int, [_vp, C.c_double, C.c_double]),
    "get_growth_factor": (C.c_double, [_vp]),
    "get_growth_rate": (C.c_double, [_vp]),
    "get_positions": (C.c_long, [_vp, _dbl_p, C.c_long]),
    "get_velocities": (C.c_long, [_vp, _dbl_p, C.c_long]),
    "get_quaternions": (C.c_long, [_vp, _dbl_p, C.c_long]),
    "get_angular_velocities": (C.c_long, [_vp, _dbl_p, C.c_long]),
    "get_inv_inertia": (C.c_long, [_vp, _dbl_p, C.c_long]),
    "get_scales": (C.c_long, [_vp, _dbl_p, C.c_long]),
    "get_masses": (C.c_long, [_vp, _dbl_p, C.c_long]),
    "step": (C.c_int, [_vp, C.c_double]),
    "step_n": (C.c_int, [_vp, C.c_double, C.c_int]),
    "counters": (C.c_int, [_vp, _vp]),
    "step_hertz": (C.c_int, [_vp, C.c_double, C.c_int, C.c_double]),
    "compute_overlaps": (C.c_int, [_vp, _dbl_p]),
    "num_particles": (C.c_int, [_vp]),
    "num_contacts": (C.c_int, [_vp]),
    "num_manifolds": (C.c_int, [_vp]),
    "max_overlap": (C.c_double, [_vp]),
    "export_lammps": (C.c_int, [_vp, C.c_char_p, C.c_int]),
    "write_vtp": (C.c_int, [_vp, C.c_char_p]),
    "get_sdf_grid": (C.c_long, [_vp, C.c_int, C.c_int, C.c_int, _dbl_p, C.c_long]),
    "export_sdf": (C.c_int, [_vp, C.c_char_p, C.c_int, C.c_int, C.c_int]),
    # diagnostics: the substep's intermediate products in the canonical order
    "debug_counts": (C.c_int, [_vp, _long_p]),
    "debug_pairs": (C.c_long, [_vp, _int_p, C.c_long]),
    "debug_contacts": (C.c_long, [_vp, _dbl_p, C.c_long]),
    "debug_contact_mu": (C.c_long, [_vp, _dbl_p, C.c_long]),
    "debug_manifolds": (C.c_long, [_vp, _dbl_p, C.c_long]),
    "debug_manifold_colors": (C.c_long, [_vp, _int_p, C.c_long]),
    "debug_contact_colors": (C.c_long, [_vp, _int_p, C.c_long]),
    "debug_lambda": (C.c_long, [_vp, _dbl_p, C.c_long]),
    "debug_pair_keys": (C.c_long, [_vp, _u64_p, C.c_long]),
    "debug_ledger": (C.c_long, [_vp, _u64_p, _dbl_p, C.c_long]),
    "debug_grounded": (C.c_long, [_vp, _int_p, C.c_long]),
    "debug_pos_lambda": (C.c_long, [_vp, _dbl_p, C.c_long]),
    "debug_hertz": (C.c_long, [_vp, _u64_p, _dbl_p, C.c_long]),
    "debug_set_max_contacts": (C.c_int, [_vp, C.c_int]),
    "debug_set_barrier_spins": (C.c_int, [_vp, C.c_long]),
    # instrumentation
    "profile_enable": (C.c_int, [_vp, C.c_int]),
    "profile_read": (C.c_int, [_vp, _dbl_p, _long_p, C.c_int, _long_p]),
    "debug_ranked": (C.c_int, [_vp, _long_p]),
    "profile_read_host": (C.c_int, [_vp, _dbl_p, C.c_int]),
    "debug_sweeps": (C.c_int, [_vp, _long_p]),
    "debug_allocs": (C.c_long, []),
    "timer_start": (C.c_int, [_vp]),
    "debug_reuse": (C.c_int, [_vp, _long_p]),
    "timer_stop": (C.c_int, [_vp, _dbl_p]),
    # batched form
    "set_scenes": (C.c_int, [_vp, C.c_int, _int_p]),
    "set_scene_material": (C.c_int, [_vp, C.c_int, C.c_double, C.c_double]),
    "set_wall_scene": (C.c_int, [_vp, C.c_int, C.c_int]),
    "scene_counters": (C.c_long, [_vp, _dbl_p, C.c_long]),
    "scene_block": (C.c_int, [_vp, _int_p, _dbl_p, C.c_int]),
    "color_block": (C.c_int, [_vp, _int_p, _dbl_p, C.c_int]),
    "device_view": (C.c_int, [_vp, C.c_int, C.POINTER(_vp), _long_p, _int_p, _int_p]),
    "get_domain": (C.c_int, [_vp, _dbl_p, _dbl_p]),
    # candidate pairs over caller-owned device arrays, with no allocation (pdem_static.cu)
    "find_pairs_static": (C.c_int, [_vp, _vp, C.c_int, C.c_double, C.c_double, _vp, C.c_long, _long_p, _vp]),
    # recorded rollout and adjoint of the XPBD substep (pdem_xadj.cu); device row pointers
    "xa_begin": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int]),
    "xa_step": (C.c_int, [_vp, C.c_double, C.c_int]),
    "xa_state": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "xa_backward": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _dbl_p]),
    "xa_info": (C.c_int, [_vp, _long_p, _dbl_p]),
    "xa_signature": (C.c_long, [_vp, _long_p, C.c_long]),
    "debug_radix_sort": (C.c_int, [_vp, _vp, C.c_int, C.c_int, _vp, _vp]),
    "xa_branches": (C.c_int, [_vp, C.POINTER(C.c_ulonglong)]),
    # forward, adjoint and tangent-linear runs of the Hertz sphere substep (pdem_adjoint.cu)
    "hz_state_size": (C.c_long, [C.c_int, C.c_int]),
    "hz_work_size": (C.c_long, [C.c_int, C.c_int]),
    "hz_contacts": (C.c_int, [C.c_int, _vp, _vp, _int_p, _vp, C.c_int, _vp, C.c_int, C.c_double, _vp, _vp, _vp,
                              C.c_long, _long_p, _vp]),
    "hz_forward": (C.c_int, [C.c_int, _vp, C.c_int, C.c_int, _vp, _vp, _vp]),
    "hz_backward": (C.c_int, [C.c_int, _vp, C.c_int, _vp, _vp, _vp, _vp, C.c_int, _vp]),
    "hz_jvp": (C.c_int, [C.c_int, _vp, C.c_int, _vp, _vp, _dbl_p, _vp, _vp]),
}


class Counters(C.Structure):
    """pdem_counters_t (include/pdem.h): the last substep's sizes, colours, sweeps and status."""
    _fields_ = [("pairs", C.c_long), ("contacts", C.c_long), ("manifolds", C.c_long),
                ("colors_velocity", C.c_int), ("colors_position", C.c_int), ("velocity_sweeps", C.c_int),
                ("stabilization_sweeps", C.c_int), ("position_sweeps", C.c_int), ("status", C.c_int),
                ("max_overlap", C.c_double), ("color_rounds_velocity", C.c_int), ("color_rounds_position", C.c_int)]


class HzModel(C.Structure):
    """pdem_hz_model (include/pdem.h): device pointers and scalars of one Hertz sphere rollout."""
    _fields_ = [("n", C.c_int), ("ncontact", C.c_int), ("nplane", C.c_int), ("contacts", _vp), ("planes", _vp),
                ("radius", _vp), ("inv_mass", _vp), ("inv_inertia", _vp), ("youngs", C.c_double),
                ("restitution", C.c_double), ("friction", C.c_double), ("poisson", C.c_double),
                ("dt", C.c_double), ("gravity", C.c_double * 3)]

STAGES = ("predict", "ghosts", "broadphase", "narrowphase", "manifolds", "colour_velocity", "warm_start",
          "velocity", "stabilization", "ledger", "friction", "integrate", "colour_position", "position",
          "commit", "hertz_pairs", "hertz_rebuild", "hertz_integrate")

_STAB_MODES = ("off", "onesided", "multilevel", "escalate", "ordered")


class CApi:
    """A loaded `<prefix>_*` library with typed entry points."""

    def __init__(self, path: str, prefix: str):
        if not os.path.exists(path):
            raise ImportError(f"C ABI library not found: {path}")
        self.path = path
        self.prefix = prefix
        self.lib = C.CDLL(path)
        self.fn = {}
        for name, (res, args) in _SIGS.items():
            sym = f"{prefix}_{name}"
            f = getattr(self.lib, sym, None)
            if f is None:
                continue
            f.restype = res
            f.argtypes = args
            self.fn[name] = f

    def has(self, name: str) -> bool:
        return name in self.fn

    def error(self) -> str:
        msg = self.fn["last_error"]()
        return msg.decode() if msg else ""

    def check(self, status: int, what: str):
        if status == OK:
            return
        msg = f"{what}: {self.error()}"
        if status == ERR_INVALID:
            raise ValueError(msg)
        raise RuntimeError(msg)


def _f64(a, cols=None):
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    if cols is not None and arr.ndim == 1 and arr.size % cols == 0:
        arr = arr.reshape(-1, cols)
    return arr


def _ptr(arr):
    return arr.ctypes.data_as(_dbl_p)


def _vec3(t):
    a = _f64(t).reshape(3)
    return a


class CApiSimulation:
    """The reference `Simulation` facade over a `<prefix>_*` C ABI.

    Method names, argument order and defaults follow src/dem_bindings.cpp:72-432. Arrays may be any
    numeric dtype; they are passed as float64. Getters return float64 (N, k) arrays for the FP64
    precision and float32 for the FP32 precision (the reference's own dtype).
    """

    def __init__(self, api: CApi, capacity: int, precision: str = "fp64"):
        if precision not in ("fp64", "fp32", "mixed"):
            raise ValueError("precision must be 'fp64', 'fp32' or 'mixed'")
        self._api = api
        self._f = api.fn
        self.precision = precision
        self._out_dtype = np.float32 if precision == "fp32" else np.float64
        code = {"fp64": 64, "fp32": 32, "mixed": PRECISION_MIXED}[precision]
        h = _vp()
        api.check(self._f["create"](int(capacity), code, C.byref(h)), "Simulation(capacity)")
        self._h = h

    # ---- lifetime -------------------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._f["destroy"](self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _call(self, name, *args):
        self._api.check(self._f[name](self._h, *args), name)

    # ---- shapes ---------------------------------------------------------------------------------
    def set_sphere_shape(self, radius):
        self._call("initialize_shape", 1, float(radius), 0.0, 0.0)

    def initialize_shape(self, shape_type, radius, height=0.0, thickness=0.0):
        self._call("initialize_shape", int(shape_type), float(radius), float(height),
                   float(thickness))

    def initialize(self, shape_type, radius=0.5, height=2.0, thickness=0.0):
        self.initialize_shape(shape_type, radius, height, thickness)

    def set_sdf_shape(self, grid, nx, ny, nz, origin, spacing, shell, inv_inertia,
                      bounding_radius):
        g = _f64(grid).ravel()
        s = _f64(shell).ravel()
        o, sp, ii = _vec3(origin), _vec3(spacing), _vec3(inv_inertia)
        self._call("set_sdf_shape", _ptr(g), int(nx), int(ny), int(nz), _ptr(o), _ptr(sp), _ptr(s),
                   int(s.size // 3), _ptr(ii), float(bounding_radius))

    def set_shell_points(self, points):
        """Replace the active shape's surface point shell (extension: seeded/stratified shells)."""
        p = _f64(points).ravel()
        self._call("set_shell_points", _ptr(p), int(p.size // 3))

    # ---- domain / global parameters --------------------------------------------------------------
    def set_domain(self, *args, **kw):
        if len(args) == 2 and not kw and np.size(args[0]) == 3:
            mn, mx = _vec3(args[0]), _vec3(args[1])
            self._call("set_domain_minmax", _ptr(mn), _ptr(mx))
            return
        if "min" in kw or "max" in kw:
            mn, mx = _vec3(kw["min"]), _vec3(kw["max"])
            self._call("set_domain_minmax", _ptr(mn), _ptr(mx))
            return
        names = ("lx", "ly", "lz", "px", "py", "pz")
        vals = dict(zip(names, args))
        vals.update(kw)
        px, py, pz = vals.get("px", True), vals.get("py", True), vals.get("pz", False)
        self._call("set_domain", float(vals["lx"]), float(vals["ly"]), float(vals["lz"]),
                   int(bool(px)), int(bool(py)), int(bool(pz)))

    def _domain(self):
        mn, mx = np.zeros(3), np.zeros(3)
        self._call("get_domain", _ptr(mn), _ptr(mx))
        return mn, mx

    def get_domain_min(self):
        """The domain minimum corner (x, y, z) (src/dem_bindings.cpp:124-125)."""
        return tuple(float(self._out_dtype(v)) for v in self._domain()[0])

    def get_domain_max(self):
        """The domain maximum corner (x, y, z) (src/dem_bindings.cpp:126-127)."""
        return tuple(float(self._out_dtype(v)) for v in self._domain()[1])

    def enable_periodicity(self, x, y, z):
        self._call("enable_periodicity", int(bool(x)), int(bool(y)), int(bool(z)))

    def set_gravity(self, gx, gy, gz):
        self._call("set_gravity", float(gx), float(gy), float(gz))

    def set_thermostat(self, temperature, tau, kB=1.0):
        self._call("set_thermostat", float(temperature), float(tau), float(kB))

    def set_solver_iterations(self, pos, vel):
        self._call("set_solver_iterations", int(pos), int(vel))

    def set_velocity_use_gs(self, use_gs):
        self._call("set_velocity_use_gs", int(bool(use_gs)))

    def set_stabilization(self, enabled):
        self.set_stabilization_mode("onesided" if enabled else "off")

    def set_stabilization_mode(self, mode):
        self._call("set_stabilization_mode", str(mode).encode())

    def set_hertz_material(self, mat, youngs, poisson):
        self._call("set_hertz_material", int(mat), float(youngs), float(poisson))

    def set_global_scale(self, s):
        self._call("set_global_scale", float(s))

    def set_dt(self, dt):
        self._call("set_dt", float(dt))

    def set_material_params(self, restitution_normal, restitution_tangent=0.0, friction=0.0):
        self._call("set_material_params", float(restitution_normal), float(restitution_tangent),
                   float(friction))

    def set_material_ids(self, ids):
        a = np.ascontiguousarray(np.asarray(ids, dtype=np.int32).ravel())
        self._call("set_material_ids", a.ctypes.data_as(_int_p), int(a.size))

    def set_pair_material(self, a, b, restitution, friction):
        self._call("set_pair_material", int(a), int(b), float(restitution), float(friction))

    def set_wall_material_id(self, wid, mat):
        self._call("set_wall_material_id", int(wid), int(mat))

    def add_plane(self, *args):
        if len(args) == 2:
            p, n = _vec3(args[0]), _vec3(args[1])
            args = (*p, *n)
        self._call("add_plane", *[float(v) for v in args])

    def add_sdf_wall(self, grid, nx, ny, nz, origin, spacing, restitution=0.0, friction=0.0):
        g = _f64(grid).ravel()
        o, sp = _vec3(origin), _vec3(spacing)
        idx = C.c_int(-1)
        self._call("add_sdf_wall", _ptr(g), int(nx), int(ny), int(nz), _ptr(o), _ptr(sp),
                   float(restitution), float(friction), C.byref(idx))
        return idx.value

    def set_wall_velocity(self, wall_index, lin_vel=(0.0, 0.0, 0.0), ang_vel=(0.0, 0.0, 0.0),
                          center=(0.0, 0.0, 0.0)):
        a, b, c = _vec3(lin_vel), _vec3(ang_vel), _vec3(center)
        self._call("set_wall_velocity", int(wall_index), _ptr(a), _ptr(b), _ptr(c))

    # ---- device-timeline timer (no reference counterpart) ------------------------------------------
    def timer_start(self):
        self._call("timer_start")

    def debug_reuse(self):
        """Substeps (since profile_enable) that kept: the manifold grouping, the contact colours,
        the manifold colours."""
        out = np.zeros(3, dtype=np.int64)
        self._call("debug_reuse", out.ctypes.data_as(_long_p))
        return {"grouping": int(out[0]), "contact_colours": int(out[1]), "manifold_colours": int(out[2])}

    def timer_stop(self):
        v = C.c_double(0.0)
        self._call("timer_stop", C.byref(v))
        return v.value

    # ---- batched form (no reference counterpart) -------------------------------------------------
    def set_scenes(self, first_body):
        """Declare scene s = bodies [first_body[s], first_body[s+1]) (call after set_positions)."""
        f = np.ascontiguousarray(first_body, dtype=np.int32)
        self._call("set_scenes", int(f.size - 1), f.ctypes.data_as(_int_p))

    def set_scene_material(self, scene, restitution, friction):
        self._call("set_scene_material", int(scene), float(restitution), float(friction))

    def set_wall_scene(self, wall, scene):
        self._call("set_wall_scene", int(wall), int(scene))

    # ---- zero-copy device arrays (src/dem_bindings.cpp:302-334) --------------------------------
    def _view(self, field, cols):
        import torch

        ptr, rows, stride, eb = _vp(), C.c_long(0), C.c_int(0), C.c_int(0)
        self._call("device_view", int(field), C.byref(ptr), C.byref(rows), C.byref(stride), C.byref(eb))

        class _DeviceArray:  # __cuda_array_interface__ v3 over the simulation's memory
            pass

        a = _DeviceArray()
        a.owner = self  # the simulation outlives the array
        shape = (rows.value, cols) if cols > 1 else (rows.value,)
        strides = (stride.value * eb.value, eb.value) if cols > 1 else (eb.value,)
        a.__cuda_array_interface__ = {"shape": shape, "strides": strides, "typestr": "<f8" if eb.value == 8 else "<f4",
                                      "data": (ptr.value or 0, False), "version": 3, "stream": None}
        return torch.as_tensor(a, device="cuda")

    def get_positions_view(self):
        """Zero-copy (N,3) device array of positions (a torch tensor aliasing the simulation's
        memory; DLPack- and __cuda_array_interface__-capable). Take it after each step."""
        return self._view(0, 3)

    def get_velocities_view(self):
        """Zero-copy (N,3) device array of velocities."""
        return self._view(1, 3)

    def get_external_forces_view(self):
        """Zero-copy (N,3) device array of the external force; writes reach the next step once
        they are complete (synchronise the writing stream before stepping)."""
        return self._view(2, 3)

    def get_inv_mass_view(self):
        """Zero-copy (N,) device array of inverse masses (read-only use)."""
        return self._view(3, 1)

    def scene_block(self):
        """The per-scene sweep block the launch shape autotuner chose (0 while tuning) and each
        candidate's mean sweep-loop time (ms per substep)."""
        b = C.c_int(0)
        ms = np.zeros(4)
        self._call("scene_block", C.byref(b), _ptr(ms), 4)
        return {"block": b.value, "candidates": [64, 128, 256, 512], "ms": ms.tolist()}

    def color_block(self):
        """The colouring launch block the batched form's autotuner chose (0 while tuning) and each
        candidate's mean colouring-launch time (ms)."""
        b = C.c_int(0)
        ms = np.zeros(3)
        self._call("color_block", C.byref(b), _ptr(ms), 3)
        return {"block": b.value, "candidates": [256, 512, 1024], "ms": ms.tolist()}

    def scene_counters(self):
        """(S, 5): max overlap, max approach, velocity / stabilization / position sweeps."""
        cap = 5 * 4096
        out = np.zeros(cap)
        n = int(self._f["scene_counters"](self._h, out.ctypes.data_as(_dbl_p), cap))
        if n < 0:
            raise RuntimeError(f"scene_counters: {self._api.error()}")
        return out[: 5 * n].reshape(n, 5)

    # ---- particle state ------------------------------------------------------------------------
    def set_positions(self, a):
        arr = np.asarray(a)
        if arr.ndim == 2 and arr.shape[1] in (3, 4):
            xyz = _f64(arr[:, :3])
            self._call("set_positions", _ptr(xyz), int(xyz.shape[0]))
            if arr.shape[1] == 4:  # column 3 is inverse mass, 0 -> 1 (src/dem_bindings.cpp:225-251)
                w = _f64(arr[:, 3])
                w = np.where(w == 0.0, 1.0, w)
                self._call("set_inv_mass", _ptr(w), int(w.size))
        else:
            xyz = _f64(arr).ravel()
            self._call("set_positions", _ptr(xyz), int(xyz.size // 3))

    def _set_rows(self, name, a, cols):
        arr = _f64(a).ravel()
        self._call(name, _ptr(arr), int(arr.size // cols))

    def set_velocities(self, a):
        self._set_rows("set_velocities", a, 3)

    def set_external_forces(self, a):
        self._set_rows("set_external_forces", a, 3)

    def clear_external_forces(self):
        self._call("clear_external_forces")

    def set_quaternions(self, a):
        self._set_rows("set_quaternions", a, 4)

    def set_angular_velocities(self, a):
        self._set_rows("set_angular_velocities", a, 3)

    def set_inv_inertia(self, a):
        self._set_rows("set_inv_inertia", a, 3)

    def set_inv_mass(self, a):
        self._set_rows("set_inv_mass", a, 1)

    def set_scales(self, a):
        self._set_rows("set_scales", a, 1)

    def set_scales_uniform(self, s):
        self._call("set_scales_uniform", float(s))

    def set_growth_params(self, rate, new_factor=-1.0):
        self._call("set_growth_params", float(rate), float(new_factor))

    def get_growth_factor(self):
        return float(self._f["get_growth_factor"](self._h))

    def get_growth_rate(self):
        return float(self._f["get_growth_rate"](self._h))

    def _get(self, name, cols, out=None):
        """Rows of a per-particle field. With `out` (an extension: a C-contiguous float64 array of at
        least n x cols values, e.g. in pinned host memory) the values are written there and a view
        of it is returned; otherwise a new array of the precision's dtype."""
        n = self.num_particles()
        if out is not None:
            buf = out.reshape(-1)
            if out.dtype != np.float64 or not out.flags.c_contiguous or buf.size < n * cols:
                raise ValueError(f"{name}: out must be C-contiguous float64 with {n * cols} values")
            got = self._f[name](self._h, _ptr(buf), int(n * cols))
            if got < 0:
                self._api.check(ERR_RUNTIME, name)
            res = buf[: min(got, n * cols)]
            return res.reshape(-1, cols) if cols > 1 else res
        buf = np.empty(n * cols, dtype=np.float64)
        got = self._f[name](self._h, _ptr(buf), int(buf.size))
        if got < 0:
            self._api.check(ERR_RUNTIME, name)
        res = buf[: min(got, buf.size)].astype(self._out_dtype)
        return res.reshape(-1, cols) if cols > 1 else res

    def get_positions(self, out=None):
        return self._get("get_positions", 3, out)

    def get_velocities(self, out=None):
        return self._get("get_velocities", 3, out)

    def get_quaternions(self, out=None):
        return self._get("get_quaternions", 4, out)

    def get_angular_velocities(self, out=None):
        return self._get("get_angular_velocities", 3, out)

    def get_inv_inertia(self):
        return self._get("get_inv_inertia", 3)

    def get_scales(self):
        return self._get("get_scales", 1)

    def get_masses(self):
        return self._get("get_masses", 1)

    # ---- stepping ------------------------------------------------------------------------------
    def step(self, dt=0.0):
        self._call("step", float(dt))

    def step_n(self, dt, n):
        """n substeps in one call across the C ABI (each exactly `step(dt)`)."""
        self._call("step_n", float(dt), int(n))

    def counters(self):
        """The last substep's P, C, M, colour counts, sweeps, error bits and max overlap."""
        c = Counters()
        self._call("counters", C.byref(c))
        return {name: getattr(c, name) for name, _ in Counters._fields_}

    def step_hertz(self, dt, substeps=1, skin_frac=0.3):
        self._call("step_hertz", float(dt), int(substeps), float(skin_frac))

    def compute_overlaps(self):
        v = C.c_double(0.0)
        self._call("compute_overlaps", C.byref(v))
        return v.value

    # ---- counters / profiling ------------------------------------------------------------------
    def num_particles(self):
        return int(self._f["num_particles"](self._h))

    def num_contacts(self):
        return int(self._f["num_contacts"](self._h))

    def num_manifolds(self):
        return int(self._f["num_manifolds"](self._h))

    def max_overlap(self):
        return float(self._f["max_overlap"](self._h))

    get_num_contacts = num_contacts
    get_num_manifolds = num_manifolds
    get_max_overlap = max_overlap

    def get_profiling_info(self):
        return {"num_particles": self.num_particles(), "num_contacts": self.num_contacts(),
                "num_manifolds": self.num_manifolds(), "max_overlap": self.max_overlap()}

    # ---- export --------------------------------------------------------------------------------
    def export_lammps(self, filename, step):
        self._call("export_lammps", os.fsencode(filename), int(step))

    def write_vtp(self, filename):
        self._call("write_vtp", os.fsencode(filename))

    def get_sdf_grid(self, resolution):
        """Packed-bed SDF over the domain (src/dem_bindings.cpp:344-355, src/output_sdf.hpp): the
        flat x-fastest field returned as a C-order (rx, ry, rz) array, as the reference does."""
        rx, ry, rz = (int(v) for v in resolution)
        out = np.zeros(max(rx * ry * rz, 0), dtype=np.float64)
        n = self._f["get_sdf_grid"](self._h, rx, ry, rz, _ptr(out), out.size)
        if n < 0:
            raise (ValueError if rx < 1 or ry < 1 or rz < 1 else RuntimeError)(f"get_sdf_grid: {self._api.error()}")
        return out.astype(self._out_dtype).reshape(rx, ry, rz)

    def export_sdf(self, filename, resolution):
        """The same field written as a VTI image (src/dem_bindings.cpp:369-376, src/io.hpp:86-110)."""
        rx, ry, rz = (int(v) for v in resolution)
        self._call("export_sdf", os.fsencode(filename), rx, ry, rz)

    # ---- diagnostics (canonical-order intermediate products of the last substep) -----------------
    def debug_counts(self):
        out = np.zeros(8, dtype=np.int64)
        self._f["debug_counts"](self._h, out.ctypes.data_as(_long_p))
        keys = ("pairs", "contacts", "manifolds", "num_bodies", "ledger", "capacity",
                "max_contacts", "pair_capacity")
        return dict(zip(keys, (int(v) for v in out)))

    def _dbg(self, name, count_key, cols, dtype=np.float64):
        n = self.debug_counts()[count_key]
        out = np.zeros(max(n * cols, 1), dtype=dtype)
        ptype = {np.float64: _dbl_p, np.int32: _int_p, np.uint64: _u64_p}[dtype]
        got = self._f[name](self._h, out.ctypes.data_as(ptype), int(out.size))
        out = out[: got * cols]
        return out.reshape(-1, cols) if cols > 1 else out

    def debug_pairs(self):
        return self._dbg("debug_pairs", "pairs", 2, np.int32)

    def debug_contacts(self):
        c = self._dbg("debug_contacts", "contacts", 17)
        mu = self._dbg("debug_contact_mu", "contacts", 1)
        return np.concatenate([c, mu.reshape(-1, 1)], axis=1) if c.size else np.zeros((0, 18))

    def debug_manifolds(self):
        return self._dbg("debug_manifolds", "manifolds", 23)

    def debug_manifold_colors(self):
        return self._dbg("debug_manifold_colors", "manifolds", 1, np.int32)

    def debug_contact_colors(self):
        return self._dbg("debug_contact_colors", "contacts", 1, np.int32)

    def debug_lambda(self):
        return self._dbg("debug_lambda", "manifolds", 4)

    def debug_pair_keys(self):
        return self._dbg("debug_pair_keys", "manifolds", 1, np.uint64)

    def debug_pos_lambda(self):
        return self._dbg("debug_pos_lambda", "contacts", 1)

    def debug_grounded(self):
        n = self.num_particles()
        out = np.zeros(max(n, 1), dtype=np.int32)
        got = self._f["debug_grounded"](self._h, out.ctypes.data_as(_int_p), int(out.size))
        return out[:got]

    def debug_ledger(self):
        n = self.debug_counts()["ledger"]
        keys = np.zeros(max(n, 1), dtype=np.uint64)
        vals = np.zeros(max(5 * n, 1), dtype=np.float64)
        got = self._f["debug_ledger"](self._h, keys.ctypes.data_as(_u64_p), _ptr(vals), int(n))
        return keys[:got], vals[: 5 * got].reshape(-1, 5)

    def debug_hertz(self, cap=1 << 24):
        keys = np.zeros(cap, dtype=np.uint64)
        xi = np.zeros(3 * cap, dtype=np.float64)
        got = self._f["debug_hertz"](self._h, keys.ctypes.data_as(_u64_p), _ptr(xi), int(cap))
        got = max(0, min(got, cap))
        return keys[:got], xi[: 3 * got].reshape(-1, 3)

    def debug_set_max_contacts(self, n):
        self._call("debug_set_max_contacts", int(n))

    def debug_set_barrier_spins(self, n):
        """Polls before a grid-barrier wait of the persistent loops gives up (0: the default)."""
        self._call("debug_set_barrier_spins", int(n))

    # ---- instrumentation -------------------------------------------------------------------------
    def profile_enable(self, on=True):
        """Start (reset) per-stage device timing and the kernel launch count."""
        self._call("profile_enable", int(bool(on)))

    def profile_read(self):
        """(dict stage -> (milliseconds, calls), kernel launches) since profile_enable."""
        ms = np.zeros(32, dtype=np.float64)
        calls = np.zeros(32, dtype=np.int64)
        launches = C.c_long(0)
        n = self._f["profile_read"](self._h, _ptr(ms), calls.ctypes.data_as(_long_p), 32, C.byref(launches))
        stages = {STAGES[i]: (float(ms[i]), int(calls[i])) for i in range(min(n, len(STAGES)))}
        return stages, int(launches.value)

    def profile_read_host(self):
        """dict stage -> host wall-clock milliseconds spent issuing it since profile_enable."""
        ms = np.zeros(32, dtype=np.float64)
        n = self._f["profile_read_host"](self._h, _ptr(ms), 32)
        return {STAGES[i]: float(ms[i]) for i in range(min(n, len(STAGES)))}

    def debug_ranked(self):
        """Substeps since profile_enable whose contact grouping was a rank scatter, and those whose
        list the scatter rejected (then sorted)."""
        out = np.zeros(2, dtype=np.int64)
        self._call("debug_ranked", out.ctypes.data_as(_long_p))
        return {"ranked": int(out[0]), "rejected": int(out[1])}

    def debug_sweeps(self):
        """Sweeps executed since profile_enable (velocity, stabilization, position) and substeps."""
        out = np.zeros(4, dtype=np.int64)
        self._call("debug_sweeps", out.ctypes.data_as(_long_p))
        return dict(zip(("velocity", "stabilization", "position", "substeps"), (int(v) for v in out)))
