"""Seeded synthetic workloads with the shapes, sizes and value distributions of the benchmark
configurations (the reference publishes no dataset; every input here is generated from a seed).

Each builder returns a `Scene`: plain NumPy arrays plus the facade calls that configure a
`Simulation` (the reference API, src/dem_bindings.cpp:72-432). Unit convention: metres, with
`set_global_scale(r_ref)` and a canonical shape radius of 1, so the narrowphase finite-difference
step (1e-4 canonical, src/narrowphase.hpp:235) is relative to the grain size.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

SPHERE, HOLLOW_CYLINDER, BOX = 1, 2, 3


@dataclass
class Scene:
    name: str
    pos: np.ndarray                      # (N,3)
    vel: np.ndarray                      # (N,3)
    inv_mass: np.ndarray                 # (N,)
    inv_inertia: np.ndarray              # (N,3)
    quat: np.ndarray | None = None       # (N,4) x,y,z,w
    angvel: np.ndarray | None = None     # (N,3)
    scales: np.ndarray | None = None     # (N,)
    shape: tuple = (SPHERE, 1.0, 0.0, 0.0)
    global_scale: float = 1.0
    domain: tuple | None = None          # (min3, max3, periodic3)
    planes: list = field(default_factory=list)
    gravity: tuple = (0.0, 0.0, -9.81)
    material: tuple = (0.5, 0.0, 0.5)    # (e_n, e_t, mu)
    iterations: tuple = (10, 10)         # (position, velocity)
    dt: float = 1e-5                     # one demStep call (= one substep)
    substeps: int = 10                   # demStep calls per outer step
    shell: np.ndarray | None = None      # optional explicit point shell
    hertz: tuple | None = None           # (E, nu) for the Hertz engine
    sdf: tuple | None = None             # set_sdf_shape arguments: a grid-SDF particle shape

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])

    def apply(self, sim):
        """Configure `sim` (any object with the reference facade methods) with this scene."""
        if self.sdf is not None:
            sim.set_sdf_shape(*self.sdf)
        else:
            sim.initialize_shape(*self.shape)
        if self.shell is not None:
            sim.set_shell_points(self.shell)
        sim.set_global_scale(self.global_scale)
        if self.domain is not None:
            mn, mx, per = self.domain
            sim.set_domain(tuple(mn), tuple(mx))
            sim.enable_periodicity(*per)
        sim.set_gravity(*self.gravity)
        sim.set_material_params(*self.material)
        sim.set_solver_iterations(*self.iterations)
        if self.hertz is not None:
            sim.set_hertz_material(0, *self.hertz)
        for p in self.planes:
            sim.add_plane(*p)
        sim.set_positions(self.pos)
        if self.quat is not None:
            sim.set_quaternions(self.quat)
        if self.scales is not None:
            sim.set_scales(self.scales)
        sim.set_velocities(self.vel)
        if self.angvel is not None:
            sim.set_angular_velocities(self.angvel)
        sim.set_inv_mass(self.inv_mass)
        sim.set_inv_inertia(self.inv_inertia)
        sim.set_dt(self.dt)
        return sim


def box_planes(mn, mx):
    """Six inward-facing planes of a closed box (point, normal)."""
    (x0, y0, z0), (x1, y1, z1) = mn, mx
    return [(x0, 0, 0, 1, 0, 0), (x1, 0, 0, -1, 0, 0), (0, y0, 0, 0, 1, 0), (0, y1, 0, 0, -1, 0),
            (0, 0, z0, 0, 0, 1), (0, 0, z1, 0, 0, -1)]


def sphere_props(radius, density):
    m = density * 4.0 / 3.0 * np.pi * radius ** 3
    inv_i = 1.0 / (0.4 * m * radius ** 2)
    return 1.0 / m, inv_i


def plain_settling(seed=1, nx=16, ny=16, nz=16, cells_z=64, radius=1e-3, spacing_r=2.2,
                   jitter_r=0.05, vmax=0.1, density=2500.0, e=0.5, mu=0.5, dt_outer=1e-4,
                   substeps=10, iterations=(10, 10)) -> Scene:
    """Plain XPBD settling: monodisperse spheres on a jittered simple-cubic lattice at the bottom of
    a closed box of nx x ny x cells_z lattice cells (6 analytic planes), uniform random velocities.
    Defaults are the 4,096-sphere configuration (16x16x16 in a 16x16x64-cell box)."""
    rng = np.random.default_rng(seed)
    a = spacing_r * radius
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    base = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1).astype(np.float64)
    # particle index runs x-fastest (i + nx*(j + ny*k)) like a poured lattice
    order = np.lexsort((base[:, 0], base[:, 1], base[:, 2]))
    base = base[order]
    pos = (base + 0.5) * a + rng.uniform(-jitter_r * radius, jitter_r * radius, base.shape)
    vel = rng.uniform(-vmax, vmax, base.shape)
    n = pos.shape[0]
    im, iI = sphere_props(radius, density)
    mn = (0.0, 0.0, 0.0)
    mx = (nx * a, ny * a, cells_z * a)
    return Scene(name=f"plain_settling_{n}", pos=pos, vel=vel, inv_mass=np.full(n, im),
                 inv_inertia=np.full((n, 3), iI), shape=(SPHERE, 1.0, 0.0, 0.0),
                 global_scale=radius, domain=(mn, mx, (False, False, False)),
                 planes=box_planes(mn, mx), gravity=(0.0, 0.0, -9.81), material=(e, 0.0, mu),
                 iterations=iterations, dt=dt_outer / substeps, substeps=substeps)


STATE_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "states")
PLAIN_SETTLED_STEPS = 800


def plain_settling_state_path(steps=PLAIN_SETTLED_STEPS):
    return os.path.join(STATE_DIR, f"plain_settling_4096_step{steps}.npz")


def plain_settled(steps=PLAIN_SETTLED_STEPS, path=None) -> Scene:
    """The 4,096-sphere settling configuration restarted from its saved state after `steps` outer
    steps (10 substeps each) of the FP64 step from the lattice start (states/make_states.py):
    positions, velocities, orientations and spins; every setting is the configuration's. The
    warm-start ledger, support levels and the restitution threshold start cold, as after any
    `set_positions`."""
    sc = plain_settling()
    st = np.load(path or plain_settling_state_path(steps))
    if st["pos"].shape != sc.pos.shape:
        raise ValueError(f"saved state holds {st['pos'].shape[0]} spheres, the configuration {sc.n}")
    sc.pos, sc.vel = st["pos"].astype(np.float64), st["vel"].astype(np.float64)
    sc.quat, sc.angvel = st["quat"].astype(np.float64), st["angvel"].astype(np.float64)
    sc.name = f"plain_settling_{sc.n}_from_step{int(st['steps'])}"
    return sc


def random_unit_quats(rng, n):
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return q


def hollow_cylinders(seed=3, n=65536, r_out=1e-3, r_in=0.6e-3, length=3e-3, box=None, fill=0.25,
                     density=1200.0, e=0.4, mu=0.3, dt_outer=5e-5, substeps=8, iterations=(20, 10),
                     shell_points=None) -> Scene:
    """Point-shell hollow cylinders (body axis y), uniform random orientations, centres by random
    sequential addition with bounding-sphere exclusion (the compiled helper) in a closed box (6
    planes). `box=None` sizes a 1 x 1 x 2 box so the bounding spheres fill `fill` of it: 65,536
    bounding spheres (radius 1.80 mm) cannot be placed without overlap in 60 x 60 x 120 mm, which
    they would fill to 3.7 times its volume."""
    rng = np.random.default_rng(seed)
    rb = float(np.hypot(r_out, 0.5 * length))  # bounding-sphere radius
    if box is None:
        side = (n * 4.0 / 3.0 * np.pi * rb ** 3 / fill / 2.0) ** (1.0 / 3.0)
        box = (side, side, 2.0 * side)
    pos, placed = rsa_spheres(seed, np.full(n, rb), (0.0, 0.0, 0.0), tuple(box))
    pos = pos[placed]
    n = pos.shape[0]
    vol = np.pi * (r_out ** 2 - r_in ** 2) * length
    m = density * vol
    term = r_out ** 2 + r_in ** 2
    ixx = m * (3 * term + length ** 2) / 12.0
    iyy = 0.5 * m * term  # body axis y
    inv_i = np.tile([1.0 / ixx, 1.0 / iyy, 1.0 / ixx], (n, 1))
    mn, mx = (0.0, 0.0, 0.0), tuple(box)
    s = r_out  # global scale: canonical outer radius 1
    return Scene(name=f"hollow_cylinders_{n}", pos=pos, vel=np.zeros((n, 3)),
                 inv_mass=np.full(n, 1.0 / m), inv_inertia=inv_i, quat=random_unit_quats(rng, n),
                 shape=(HOLLOW_CYLINDER, 1.0, length / s, (r_out - r_in) / s), global_scale=s,
                 domain=(mn, mx, (False, False, False)), planes=box_planes(mn, mx),
                 material=(e, 0.0, mu), iterations=iterations, dt=dt_outer / substeps,
                 substeps=substeps, shell=shell_points)


def deposit(sc: Scene, dem, outer_steps, v_down=0.5, precision="fp64", dt_scale=1.0) -> Scene:
    """The scene after a gravity deposition: every body starts with `v_down` m/s along gravity on
    top of its own velocity and the scene is stepped `outer_steps` outer steps of its substeps, each
    of dt_scale times its dt (a preparation run may take longer substeps than the configuration),
    by `dem.Simulation` in `precision`. Returns a copy whose positions, velocities, orientations and
    spins are the end state; its own dt is unchanged."""
    import copy
    g = np.asarray(sc.gravity, dtype=np.float64)
    gn = np.linalg.norm(g)
    out = copy.copy(sc)
    out.vel = sc.vel + (v_down * g / gn if gn > 0 else 0.0)
    sim = out.apply(dem.Simulation(sc.n + 8, precision))
    for _ in range(outer_steps):
        for _ in range(sc.substeps):
            sim.step(sc.dt * dt_scale)
    out.pos, out.vel = sim.get_positions(), sim.get_velocities()
    out.quat, out.angvel = sim.get_quaternions(), sim.get_angular_velocities()
    out.name = f"{sc.name}_deposited{outer_steps}"
    sim.close()
    return out


_RSA_SRC = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_gen", "rsa.c")
_RSA_LIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_gen", "librsa.so")


def _rsa_lib():
    if not os.path.exists(_RSA_LIB) or os.path.getmtime(_RSA_LIB) < os.path.getmtime(_RSA_SRC):
        subprocess.run(["gcc", "-O2", "-shared", "-fPIC", "-o", _RSA_LIB, _RSA_SRC, "-lm"], check=True)
    lib = ctypes.CDLL(_RSA_LIB)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.pdem_rsa_spheres.restype = ctypes.c_long
    lib.pdem_rsa_spheres.argtypes = [ctypes.c_long, dp, dp, dp, ctypes.POINTER(ctypes.c_int),
                                     ctypes.c_ulonglong, ctypes.c_int, dp,
                                     ctypes.POINTER(ctypes.c_ubyte)]
    lib.pdem_rsa_spheres_region.restype = ctypes.c_long
    lib.pdem_rsa_spheres_region.argtypes = [ctypes.c_long, dp, dp, dp, ctypes.c_ulonglong, ctypes.c_int,
                                            ctypes.c_int, dp, dp, ctypes.POINTER(ctypes.c_ubyte)]
    return lib


def rsa_spheres(seed, radii, lo, hi, periodic=(False, False, False), tries=1000):
    """Random sequential addition (largest first, uniform proposals, rejection on overlap) by the
    compiled helper _gen/rsa.c; returns (positions, placed mask)."""
    lib = _rsa_lib()
    r = np.ascontiguousarray(radii, dtype=np.float64)
    order = np.argsort(-r, kind="stable")
    rs = np.ascontiguousarray(r[order])
    pos = np.zeros((r.size, 3))
    placed = np.zeros(r.size, dtype=np.uint8)
    lo = np.ascontiguousarray(lo, dtype=np.float64)
    hi = np.ascontiguousarray(hi, dtype=np.float64)
    per = np.ascontiguousarray(np.asarray(periodic, dtype=np.int32))
    dp = ctypes.POINTER(ctypes.c_double)
    lib.pdem_rsa_spheres(r.size, rs.ctypes.data_as(dp), lo.ctypes.data_as(dp), hi.ctypes.data_as(dp),
                         per.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), int(seed), int(tries),
                         pos.ctypes.data_as(dp), placed.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)))
    out = np.zeros_like(pos)
    ok = np.zeros(r.size, dtype=bool)
    out[order] = pos
    ok[order] = placed.astype(bool)
    return out, ok


def polydisperse(seed=2, n=262144, median=1e-3, sigma=0.25, rmin=0.5e-3, rmax=2e-3, phi=0.35,
                 density=2500.0, E=1e7, nu=0.3, mu=0.4, e=0.6, dt_outer=2e-5, substeps=10,
                 periodic=True) -> Scene:
    """Polydisperse lognormal spheres (median 1 mm, sigma 0.25, clipped to [0.5, 2] mm) placed
    without overlap by random sequential addition in a box periodic in x and y with a floor plane
    at z = 0; L_x = L_y and the height 2 L_x are chosen for a solids fraction `phi`."""
    rng = np.random.default_rng(seed)
    r = np.clip(rng.lognormal(np.log(median), sigma, n), rmin, rmax)
    vs = np.sum(4.0 / 3.0 * np.pi * r ** 3)
    L = (vs / (2.0 * phi)) ** (1.0 / 3.0)
    H = 2.0 * L
    pos, placed = rsa_spheres(seed, r, (0.0, 0.0, 0.0), (L, L, H), (periodic, periodic, False))
    keep = np.nonzero(placed)[0]
    pos, r = pos[keep], r[keep]
    n = pos.shape[0]
    m = density * 4.0 / 3.0 * np.pi * r ** 3
    inv_i = 1.0 / (0.4 * m * r ** 2)
    mn, mx = (0.0, 0.0, 0.0), (L, L, H)
    return Scene(name=f"polydisperse_{n}", pos=pos, vel=np.zeros((n, 3)), inv_mass=1.0 / m,
                 inv_inertia=np.repeat(inv_i[:, None], 3, axis=1), scales=r / median,
                 shape=(SPHERE, 1.0, 0.0, 0.0), global_scale=median,
                 domain=(mn, mx, (periodic, periodic, False)),
                 planes=[(0.0, 0.0, 0.0, 0.0, 0.0, 1.0)], material=(e, 0.0, mu),
                 dt=dt_outer / substeps, substeps=substeps, hertz=(E, nu))


# ---------------------------------------------------------------------------------------------
# batched rotating drums
def drum_wall_grid(R=6e-3, length=4e-3, h=0.5e-3):
    """Hollow-cylinder container (axis z) as a world-space SDF grid, positive in the void."""
    nx = ny = int(np.ceil(2.4 * R / h)) + 1
    nz = int(np.ceil((length + 4 * h) / h)) + 1
    origin = np.array([-1.2 * R, -1.2 * R, -2 * h])
    x = origin[0] + h * np.arange(nx)
    y = origin[1] + h * np.arange(ny)
    z = origin[2] + h * np.arange(nz)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    radial = R - np.sqrt(X ** 2 + Y ** 2)
    axial = np.minimum(Z, length - Z)
    grid = np.minimum(radial, axial)  # x-fastest after ravel of (z, y, x)
    return grid.ravel(), nx, ny, nz, origin, (h, h, h)


def drum_deposit(seed, radii, R, length, tries=200):
    """Random sequential addition of the spheres into the lower half (y <= 0) of a drum of radius R
    and length `length` (axis z); returns (positions, placed mask)."""
    lib = _rsa_lib()
    r = np.ascontiguousarray(radii, dtype=np.float64)
    order = np.argsort(-r, kind="stable")
    rs = np.ascontiguousarray(r[order])
    pos = np.zeros((r.size, 3))
    placed = np.zeros(r.size, dtype=np.uint8)
    lo = np.array([-R, -R, 0.0])
    hi = np.array([R, 0.0, length])
    rg = np.array([R, 0.0, 0.0, 0.0])
    dp = ctypes.POINTER(ctypes.c_double)
    lib.pdem_rsa_spheres_region(r.size, rs.ctypes.data_as(dp), lo.ctypes.data_as(dp), hi.ctypes.data_as(dp),
                                int(seed), int(tries), 1, rg.ctypes.data_as(dp), pos.ctypes.data_as(dp),
                                placed.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)))
    out = np.zeros_like(pos)
    ok = np.zeros(r.size, dtype=bool)
    out[order] = pos
    ok[order] = placed.astype(bool)
    return out, ok


def rotating_drums(seed=4, scenes=512, R=50e-3, length=20e-3, nmin=256, nmax=8192, rlo=0.8e-3, rhi=1.2e-3,
                   fill=0.30, density=2500.0, dt_outer=5e-5, substeps=10, grid_h=1e-3):
    """Batched rotating drums (one scene per drum): omega ~ U[0.5, 3] rad/s about the drum axis (z),
    N_s ~ U{nmin..nmax} spheres with radii ~ U[rlo, rhi], mu ~ U[0.2, 0.8], e ~ U[0.3, 0.9], placed by
    seeded random deposition in the lower half of the drum up to `fill` of the half volume (capped
    at N_s). Gravity -9.81 m/s^2 along y. Returns (scenes, extras) for batch.apply_batch; every
    drum is the same container grid (shared on the device), turning at its own rate."""
    rng = np.random.default_rng(seed)
    grid = drum_wall_grid(R, length, grid_h)
    half_volume = 0.5 * np.pi * R * R * length
    out, extras = [], []
    for s in range(scenes):
        omega = rng.uniform(0.5, 3.0)
        ns = int(rng.integers(nmin, nmax + 1))
        mu = rng.uniform(0.2, 0.8)
        e = rng.uniform(0.3, 0.9)
        r = rng.uniform(rlo, rhi, ns)
        vol = np.cumsum(4.0 / 3.0 * np.pi * r ** 3)
        r = r[: max(1, int(np.searchsorted(vol, fill * half_volume)))]
        pos, ok = drum_deposit(int(rng.integers(1 << 62)), r, R, length)
        r, pos = r[ok], pos[ok]
        m = density * 4.0 / 3.0 * np.pi * r ** 3
        iI = 1.0 / (0.4 * m * r ** 2)
        out.append(Scene(name=f"drum{s}", pos=pos, vel=np.zeros_like(pos), inv_mass=1.0 / m,
                         inv_inertia=np.repeat(iI[:, None], 3, 1), scales=r / 1e-3, global_scale=1e-3,
                         domain=((-R, -R, 0.0), (R, R, length), (False, False, False)),
                         gravity=(0.0, -9.81, 0.0), material=(e, 0.0, mu), iterations=(10, 10),
                         dt=dt_outer / substeps, substeps=substeps))

        def extra(sim, w=omega):
            wid = sim.add_sdf_wall(*grid, 0.5, 0.5)
            sim.set_wall_velocity(wid, (0.0, 0.0, 0.0), (0.0, 0.0, w), (0.0, 0.0, 0.0))
        extras.append(extra)
    return out, extras


def calibration_boxes(seed=5, scenes=64, per_scene=2048, radius=1e-3, box=(40e-3, 40e-3, 80e-3),
                      lattice=(8, 8, 32), jitter=0.1e-3, vmax=0.2, density=2500.0):
    """Differentiable-calibration workload: `scenes` independent boxes (six planes shared by every
    scene) of `per_scene` spheres of radius `radius`, each on a lattice of `lattice` cells filling
    the box with seeded jitter, initial velocities uniform in +-vmax, no spin.
    Returns dict(x0, v0, w0 (n, 3); r, m, I (n,); first (scenes + 1); planes (6 x 6))."""
    nx, ny, nz = lattice
    if nx * ny * nz != per_scene:
        raise ValueError("lattice cells must equal the spheres per scene")
    rng = np.random.default_rng(seed)
    h = np.array(box) / np.array(lattice)
    cells = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"), -1).reshape(-1, 3)
    base = (cells + 0.5) * h
    xs = [base + rng.uniform(-jitter, jitter, base.shape) for _ in range(scenes)]
    n = scenes * per_scene
    r = np.full(n, radius)
    m = density * 4.0 / 3.0 * np.pi * r ** 3
    (x1, y1, z1) = box
    planes = [[0, 0, 0, 1, 0, 0], [x1, 0, 0, -1, 0, 0], [0, 0, 0, 0, 1, 0], [0, y1, 0, 0, -1, 0],
              [0, 0, 0, 0, 0, 1], [0, 0, z1, 0, 0, -1]]
    return dict(x0=np.concatenate(xs), v0=rng.uniform(-vmax, vmax, (n, 3)), w0=np.zeros((n, 3)), r=r, m=m,
                I=0.4 * m * r * r, first=np.arange(scenes + 1) * per_scene, planes=planes)


def calibration_box_scene(index=0, material=(0.6, 0.0, 0.3), dt=2e-5, **kw):
    """Box `index` of `calibration_boxes` (2048 spheres on a jittered lattice, velocities uniform in
    +-0.2 m/s) as a Scene for the plain XPBD step: six planes, gravity, the given material
    (e_n, e_t, mu), substep dt, iterations (10, 10)."""
    c = calibration_boxes(**kw)
    lo, hi = c["first"][index], c["first"][index + 1]
    r = float(c["r"][lo])
    im, iI = 1.0 / c["m"][lo:hi], 1.0 / c["I"][lo:hi]
    pl = [tuple(p) for p in c["planes"]]
    box = (pl[1][0], pl[3][1], pl[5][2])
    return Scene(name=f"calibration_box_{index}", pos=c["x0"][lo:hi].copy(), vel=c["v0"][lo:hi].copy(),
                 inv_mass=im, inv_inertia=np.repeat(iI[:, None], 3, axis=1), angvel=c["w0"][lo:hi].copy(),
                 global_scale=r, domain=((0.0, 0.0, 0.0), box, (False, False, False)), planes=pl,
                 material=tuple(material), iterations=(10, 10), dt=dt)


def hollow_cylinder_shell(n=512, seed=3, r_out=1.0, r_in=0.6, length=3.0):
    """Seeded stratified point shell of a hollow cylinder (body axis y, canonical units), for
    `set_shell_points`: points on the outer and inner lateral surfaces and the two annular caps,
    allotted by area; on each surface the parameter square is cut into one stratum per point
    (angle-major rows) and each point is jittered uniformly inside its stratum; the caps are
    sampled uniformly in area (radius from the square root of a uniform in r^2)."""
    rng = np.random.default_rng(seed)
    areas = np.array([2 * np.pi * r_out * length, 2 * np.pi * r_in * length,
                      np.pi * (r_out ** 2 - r_in ** 2), np.pi * (r_out ** 2 - r_in ** 2)])
    counts = np.floor(n * areas / areas.sum()).astype(int)
    for k in np.argsort(-(n * areas / areas.sum() - counts))[: n - counts.sum()]:
        counts[k] += 1

    def strata(m, aspect):
        """m jittered points in [0, 1)^2 on a rows x cols grid of strata near the given aspect."""
        cols = max(1, int(round(np.sqrt(m * aspect))))
        rows = -(-m // cols)
        cells = np.arange(rows * cols)
        keep = np.sort(rng.permutation(cells)[:m])
        u = (keep % cols + rng.uniform(0, 1, m)) / cols
        v = (keep // cols + rng.uniform(0, 1, m)) / rows
        return u, v

    pts = []
    for k, (m, rad) in enumerate(zip(counts[:2], (r_out, r_in))):
        u, v = strata(m, 2 * np.pi * rad / length)
        th = 2 * np.pi * u
        pts.append(np.stack([rad * np.cos(th), (v - 0.5) * length, rad * np.sin(th)], 1))
    for m, y in zip(counts[2:], (0.5 * length, -0.5 * length)):
        u, v = strata(m, 2 * np.pi * 0.8 / (r_out - r_in))
        th = 2 * np.pi * u
        rr = np.sqrt(r_in ** 2 + v * (r_out ** 2 - r_in ** 2))
        pts.append(np.stack([rr * np.cos(th), np.full(m, y), rr * np.sin(th)], 1))
    return np.concatenate(pts)


def box_wall_grid(L, H, h=2e-3, pad=2):
    """An open-top box [0, L]^2 x [0, H] as one world-space SDF grid wall (positive inside: the
    distance to the nearest of the floor and the four sides), for engines that take no planes."""
    nx = ny = int(np.ceil(L / h)) + 1 + 2 * pad
    nz = int(np.ceil(H / h)) + 1 + 2 * pad
    origin = np.array([-pad * h, -pad * h, -pad * h])
    x = origin[0] + h * np.arange(nx)
    y = origin[1] + h * np.arange(ny)
    z = origin[2] + h * np.arange(nz)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    grid = np.minimum.reduce([Z, X, L - X, Y, L - Y])  # x-fastest after ravel of (z, y, x)
    return grid.ravel(), nx, ny, nz, origin, (h, h, h)


def polydisperse_hertz_closed(seed=2, n=262144, **kw):
    """The polydisperse packing for the Hertz engine, closed: the reference's engine refuses
    periodic domains and analytic planes, so the box is closed in x and y and its floor and sides
    are one SDF grid wall. Returns (scene, extra) where extra(sim) adds the wall."""
    sc = polydisperse(seed=seed, n=n, periodic=False, **kw)
    (mn, mx, _) = sc.domain
    L, H = mx[0], mx[2]
    sc.planes = []
    grid = box_wall_grid(L, H)

    def extra(sim):
        sim.add_sdf_wall(*grid, sc.material[0], sc.material[2])
    return sc, extra
