"""The reference's physical acceptance checks, run on the B200 step through the public facade.

The reference validates its solvers with analytic known answers rather than stored vectors. The same
checks, restated here with the same set-ups and pass bars:

* coloured Gauss-Seidel XPBD step (test_colored_gs.py:42-107, gate :147):
  - binary restitution: a lone head-on collision of equal spheres realises the prescribed
    restitution, |e_eff - e| < 0.03 with e_eff = sqrt(KE_after / KE_before), and keeps the total
    momentum (drift < 1e-4), for e = 0.2, 0.5, 0.8, 0.95;
  - conservation: a cloud of hollow cylinders fired at each other in free space (off-centre
    contacts that spin them up) keeps its total linear momentum; its angular momentum drift is
    reported by the reference without a bar and is bounded here loosely;
* Hertz-Mindlin engine (test_hertz.py:27-115):
  - binary restitution from the damping formula, |e_eff - e| < 0.04 for e = 0.2, 0.5, 0.8;
  - a slab of locked spheres on a grid-SDF floor under tilted gravity sticks at mu = 0.9
    (|slide| < 1) and slides at mu = 0.05 (slide > 5);
  - kinetic Coulomb slide of one locked sphere: distance within 10 % (mu 0.3) and 15 % (mu 0.6) of
    0.5 (g_x - mu g_z) t^2;
  - slide-to-roll: a sphere launched sliding ends rolling at v / v0 = 5/7 (within 0.03) and
    w r / v0 = 5/7 (within 0.05).
"""
import numpy as np
import pytest

from peclet.dem._capi import CApiSimulation

pytestmark = pytest.mark.gpu


def _sim(api, n, precision):
    return CApiSimulation(api, n, precision)


# ------------------------------------------------------------------ coloured GS (XPBD step)
def _binary(api, e, precision):
    r, u, dt = 0.5, 1.0, 0.005
    s = _sim(api, 2, precision)
    s.initialize(shape_type=1, radius=r)
    s.set_sphere_shape(r)
    s.set_domain((-10, -10, -10), (10, 10, 10))
    s.set_gravity(0, 0, 0)
    s.set_material_params(e, 0.0, 0.0)
    s.set_solver_iterations(10, 12)
    s.set_dt(dt)
    s.set_velocity_use_gs(True)
    s.set_positions(np.array([[-2.0, 0, 0, 1.0], [2.0, 0, 0, 1.0]]))  # column 3: inverse mass 1
    v = np.array([[u, 0, 0], [-u, 0, 0]], dtype=np.float64)
    s.set_velocities(v)
    ke0 = 0.5 * (v ** 2).sum()
    for _ in range(1200):
        s.step(dt)
    vf = s.get_velocities()[:2]
    ke1 = 0.5 * (vf ** 2).sum()
    s.close()
    return np.sqrt(max(ke1, 0.0) / ke0), np.abs(vf.sum(0)).max()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("e", [0.2, 0.5, 0.8, 0.95])
def test_binary_restitution_colored_gs(gpu_api, precision, e):
    eff, drift = _binary(gpu_api, e, precision)
    assert abs(eff - e) < 0.03, f"e={e}: e_eff={eff}"
    assert drift < 1e-4


def _rot(q):
    x, y, z, w = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    R = np.empty((len(q), 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_momentum_conservation_cylinder_cloud(gpu_api, precision):
    n, dt = 24, 0.004
    s = _sim(gpu_api, n, precision)
    s.initialize(shape_type=2, radius=0.5, height=1.0, thickness=0.2)
    s.set_domain((-20, -20, -20), (20, 20, 20))
    s.set_gravity(0, 0, 0)
    s.set_material_params(0.7, 0.0, 0.0)
    s.set_solver_iterations(8, 10)
    s.set_dt(dt)
    s.set_velocity_use_gs(True)
    rng = np.random.default_rng(0)
    p0 = rng.uniform(-3, 3, (n, 3))
    s.set_positions(np.c_[p0, np.ones(n)])  # unit mass
    vel = rng.normal(0, 2.0, (n, 3))
    s.set_velocities(vel)
    s.set_quaternions(np.tile([0.0, 0.0, 0.0, 1.0], (n, 1)))
    s.set_angular_velocities(np.zeros((n, 3)))
    s.set_scales(np.ones(n))
    inv_i = s.get_inv_inertia()[:n, :3]
    i_loc = np.where(inv_i > 0, 1.0 / np.maximum(inv_i, 1e-30), 0.0)

    def momenta():
        x, v = s.get_positions()[:n], s.get_velocities()[:n]
        w, R = s.get_angular_velocities()[:n], _rot(s.get_quaternions()[:n])
        spin = np.einsum("nij,nj->ni", R, i_loc * np.einsum("nji,nj->ni", R, w))
        li = np.cross(x, v) + spin
        return v.sum(0), li.sum(0), np.linalg.norm(li, axis=1).sum()

    p_init, l_init, _ = momenta()
    l_scale, spun = 1e-30, 0.0
    for i in range(500):
        s.step(dt)
        if i == 250:
            spun = np.abs(s.get_angular_velocities()[:n]).max()
        l_scale = max(l_scale, momenta()[2])
    p_fin, l_fin, _ = momenta()
    s.close()
    p_drift = np.linalg.norm(p_fin - p_init) / np.abs(vel).sum()
    l_drift = np.linalg.norm(l_fin - l_init) / l_scale
    assert spun > 0.0  # off-centre contacts imparted spin
    assert p_drift < (1e-10 if precision == "fp64" else 1e-5), p_drift
    assert l_drift < 0.05, l_drift


# ------------------------------------------------------------------ Hertz-Mindlin engine
E0, NU0, DT = 1.0e7, 0.25, 5e-5


def _floor_grid(lo, hi, res):
    """The floor z = 0 as a world-space grid SDF (positive above), nodes spanning [lo, hi]."""
    nx, ny, nz = res
    z = np.linspace(lo[2], hi[2], nz)
    grid = np.broadcast_to(z[:, None, None], (nz, ny, nx)).ravel()  # x fastest
    spacing = tuple((np.asarray(hi, float) - np.asarray(lo, float)) / (np.asarray(res) - 1))
    return np.ascontiguousarray(grid), nx, ny, nz, tuple(lo), spacing


def _hertz_base(api, n, lo, hi, e, mu, precision):
    s = _sim(api, n, precision)
    s.set_sphere_shape(0.5)
    s.set_domain(lo, hi)
    s.enable_periodicity(False, False, False)
    s.set_material_params(e, 0.0, mu)
    s.set_hertz_material(0, E0, NU0)
    s.set_thermostat(0, 0)
    return s


def _hertz_binary(api, e, precision):
    s = _hertz_base(api, 2, (0, 0, 0), (20, 20, 20), e, 0.0, precision)
    s.set_positions(np.array([[8.0, 10, 10], [12, 10, 10]]))
    s.set_scales_uniform(1.0)
    s.set_inv_mass(np.ones(2))
    s.set_inv_inertia(np.full((2, 3), 1.0))
    s.set_velocities(np.array([[1.0, 0, 0], [-1, 0, 0]]))
    s.set_gravity(0, 0, 0)
    s.step_hertz(DT, 60000)
    v = s.get_velocities()
    s.close()
    return (v[1, 0] - v[0, 0]) / 2.0


@pytest.mark.parametrize("e", [0.2, 0.5, 0.8])
def test_hertz_binary_restitution(gpu_api, e):
    assert abs(_hertz_binary(gpu_api, e, "fp64") - e) < 0.04


def _slab(api, mu, steps=200000):
    pts = np.array([(4 + 1.9 * i, 4 + 1.9 * j, 0.55 + 1.9 * k) for i in range(4) for j in range(4) for k in range(2)])
    n = len(pts)
    lo, hi = (0, 0, -1.0), (60, 12, 8)
    s = _hertz_base(api, n, lo, hi, 0.2, mu, "fp64")
    s.add_sdf_wall(*_floor_grid(lo, hi, (96, 24, 24)), 0.2, mu)
    s.set_positions(pts)
    s.set_scales_uniform(1.0)
    s.set_inv_mass(np.ones(n))
    s.set_inv_inertia(np.zeros((n, 3)))  # rotation locked
    s.set_velocities(np.zeros((n, 3)))
    s.set_gravity(5.0, 0.0, -10.0)
    s.step_hertz(DT, steps)
    d = float(s.get_positions()[:, 0].mean() - pts[:, 0].mean())
    s.close()
    return d


def test_hertz_slab_stick_and_slip(gpu_api):
    assert abs(_slab(gpu_api, 0.9)) < 1.0
    assert _slab(gpu_api, 0.05) > 5.0


def _single(api, mu, gx=8.0, steps=160000, v0=0.0, inv_i=0.0):
    lo, hi = (0, 0, -1.0), (200, 8, 6)
    s = _hertz_base(api, 1, lo, hi, 0.0, mu, "fp64")
    s.add_sdf_wall(*_floor_grid(lo, hi, (128, 16, 16)), 0.0, mu)
    s.set_positions(np.array([[5.0, 4, 0.5]]))
    s.set_scales_uniform(1.0)
    s.set_inv_mass(np.ones(1))
    s.set_inv_inertia(np.full((1, 3), inv_i))
    s.set_velocities(np.array([[v0, 0, 0]]))
    s.set_gravity(gx, 0.0, -10.0)
    s.step_hertz(DT, steps)
    x, v, w = s.get_positions()[0], s.get_velocities()[0], s.get_angular_velocities()[0]
    s.close()
    return x, v, w


def test_hertz_kinetic_slide(gpu_api):
    t = 160000 * DT
    d3 = _single(gpu_api, 0.3)[0][0] - 5.0
    d6 = _single(gpu_api, 0.6)[0][0] - 5.0
    assert abs(d3 / (0.5 * 5 * t * t) - 1) < 0.1
    assert abs(d6 / (0.5 * 2 * t * t) - 1) < 0.15


def test_hertz_slide_to_roll(gpu_api):
    v0 = 4.0
    _, v, w = _single(gpu_api, 0.5, gx=0.0, steps=120000, v0=v0, inv_i=1.0 / (0.4 * 0.25))
    assert abs(v[0] / v0 - 5 / 7) < 0.03
    assert abs(w[1] * 0.5 / v0 - 5 / 7) < 0.05
