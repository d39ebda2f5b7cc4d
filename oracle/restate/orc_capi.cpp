// C API of the oracle restatement (test infrastructure, never shipped).
//
// Exposes orc::Sim<float> / orc::Sim<double> behind the same `<prefix>_*` ABI as the B200 library
// (include/pdem.h), with prefix `orc`, so the parity tests drive the oracle and the GPU through one
// Python facade. Precision 32 restates the reference's float arithmetic; 64 is the FP64 oracle;
// 65 is the FP64 oracle on forward-mode dual numbers (orc_dual.hpp): the same value run, with
// tangents seeded by orc_dual_seed and read by orc_dual_get (the adjoint's forward-mode check).
#include <cstring>
#include <exception>
#include <stdexcept>
#include <string>
#include <vector>

#include "orc_dual.hpp"  // before the oracle: its std:: overloads must be visible to the templates
#include "orc_sim.hpp"

namespace {
thread_local std::string g_err;

struct Handle {
  orc::Sim<float>* f = nullptr;
  orc::Sim<double>* d = nullptr;
  orc::Sim<orc::Dual>* x = nullptr;
};

template <class F>
int with(void* h, F&& fn) {
  try {
    Handle* H = static_cast<Handle*>(h);
    if (H->f)
      fn(*H->f);
    else if (H->x)
      fn(*H->x);
    else
      fn(*H->d);
    return 0;
  } catch (const std::invalid_argument& e) {
    g_err = e.what();
    return 2;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}
// a value as double (the value part of a dual number)
inline double dv(double x) { return x; }
inline double dv(float x) { return x; }
inline double dv(const orc::Dual& x) { return x.v; }
template <class R>
std::vector<R> vec(const double* p, long n) {
  std::vector<R> v(n > 0 ? n : 0);
  for (long i = 0; i < n; ++i)
    v[i] = static_cast<R>(p[i]);
  return v;
}
template <class R>
orc::V3<R> v3(const double* p) {
  return orc::V3<R>{(R)p[0], (R)p[1], (R)p[2]};
}
}  // namespace

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

int orc_create(int capacity, int precision, void** out) {
  try {
    Handle* H = new Handle;
    if (precision == 32)
      H->f = new orc::Sim<float>(capacity);
    else if (precision == 65)
      H->x = new orc::Sim<orc::Dual>(capacity);
    else
      H->d = new orc::Sim<double>(capacity);
    *out = H;
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}
void orc_destroy(void* h) {
  Handle* H = static_cast<Handle*>(h);
  delete H->f;
  delete H->d;
  delete H->x;
  delete H;
}

int orc_initialize_shape(void* h, int type, double r, double height, double thick) {
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    S.initializeShape(type, (R)r, (R)height, (R)thick);
  });
}
int orc_set_sdf_shape(void* h, const double* grid, int nx, int ny, int nz, const double* origin,
                      const double* spacing, const double* shell, int nshell, const double* invI,
                      double bR) {
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    S.setSdfShape(vec<R>(grid, (long)nx * ny * nz), nx, ny, nz, v3<R>(origin), v3<R>(spacing),
                  vec<R>(shell, (long)nshell * 3), v3<R>(invI), (R)bR);
  });
}
int orc_set_shell_points(void* h, const double* pts, int n) {
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    S.setShellPoints(vec<R>(pts, (long)n * 3));
  });
}
int orc_set_domain(void* h, double lx, double ly, double lz, int px, int py, int pz) {
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    S.setDomain((R)lx, (R)ly, (R)lz, px, py, pz);
  });
}
int orc_set_domain_minmax(void* h, const double* mn, const double* mx) {
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    S.setDomainMinMax(v3<R>(mn), v3<R>(mx));
  });
}
int orc_enable_periodicity(void* h, int x, int y, int z) {
  return with(h, [&](auto& S) {
    S.px = x;
    S.py = y;
    S.pz = z;
  });
}
int orc_set_gravity(void* h, double gx, double gy, double gz) {
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    S.gravity = {(R)gx, (R)gy, (R)gz};
  });
}
int orc_set_thermostat(void* h, double T, double tau, double kB) {
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    S.thermoTemp = (R)T;
    S.thermoTau = (R)tau;
    S.thermoKB = (R)kB;
  });
}
int orc_set_solver_iterations(void* h, int pos, int vel) {
  return with(h, [&](auto& S) {
    S.posIters = pos;
    S.velIters = vel;
  });
}
int orc_set_velocity_use_gs(void* h, int b) {
  return with(h, [&](auto& S) { S.useGS = b != 0; });
}
int orc_set_stabilization_mode(void* h, const char* mode) {
  return with(h, [&](auto& S) {
    const std::string m(mode);
    if (m == "off")
      S.stabMode = 0;
    else if (m == "onesided")
      S.stabMode = 1;
    else if (m == "multilevel")
      S.stabMode = 2;
    else if (m == "escalate")
      S.stabMode = 3;
    else if (m == "ordered")
      S.stabMode = 4;
    else
      throw std::invalid_argument(
          "set_stabilization_mode: expected 'off', 'onesided', 'multilevel', 'escalate' or 'ordered'");
  });
}
int orc_set_hertz_material(void* h, int mat, double E, double nu) {
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    if (mat < 0 || mat >= 8)
      throw std::invalid_argument("material id out of range");
    S.hzE[mat] = (R)E;
    S.hzNu[mat] = (R)nu;
  });
}
int orc_set_global_scale(void* h, double s) {
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    S.globalScale = (R)s;
    S.skin = R(0.1) * (R)s;
  });
}
int orc_set_dt(void* h, double dt) {
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    S.dt = (R)dt;
  });
}
int orc_set_material_params(void* h, double en, double et, double mu) {
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    S.eN = (R)en;
    S.mu = (R)mu;
    S.eT = (R)et;
  });
}
int orc_set_material_ids(void* h, const int* ids, int n) {
  return with(h, [&](auto& S) {
    for (int i = 0; i < S.numReal && i < n; ++i)
      S.materialId[i] = (unsigned char)ids[i];
  });
}
int orc_set_pair_material(void* h, int a, int b, double e, double mu) {
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    S.setPairMaterial(a, b, (R)e, (R)mu);
  });
}
int orc_set_wall_material_id(void* h, int wid, int mat) {
  return with(h, [&](auto& S) {
    if (wid < 0 || wid >= (int)S.walls.size())
      throw std::invalid_argument("wall index out of range");
    S.walls[wid].materialId = mat;
  });
}
int orc_add_plane(void* h, double px, double py, double pz, double nx, double ny, double nz) {
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    S.addPlane({(R)px, (R)py, (R)pz}, {(R)nx, (R)ny, (R)nz});
  });
}
int orc_add_sdf_wall(void* h, const double* grid, int nx, int ny, int nz, const double* origin,
                     const double* spacing, double e, double mu, int* outIdx) {
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    *outIdx = S.addSdfWall(vec<R>(grid, (long)nx * ny * nz), nx, ny, nz, v3<R>(origin),
                           v3<R>(spacing), (R)e, (R)mu);
  });
}
int orc_set_wall_velocity(void* h, int idx, const double* lin, const double* ang,
                          const double* center) {
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    if (idx < 0 || idx >= (int)S.walls.size())
      throw std::runtime_error("setWallVelocity: wall index out of range");
    S.walls[idx].linVel = v3<R>(lin);
    S.walls[idx].angVel = v3<R>(ang);
    S.walls[idx].center = v3<R>(center);
  });
}
int orc_set_positions(void* h, const double* xyz, int n) {
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    S.setPositions(vec<R>(xyz, (long)n * 3));
  });
}
#define ORC_SET3(NAME, FIELD)                                                     \
  int orc_##NAME(void* h, const double* a, int n) {                               \
    return with(h, [&](auto& S) {                                                 \
      using R = decltype(S.dt);                                                   \
      for (int i = 0; i < S.numReal && i < n; ++i)                                \
        S.FIELD[i] = {(R)a[3 * i], (R)a[3 * i + 1], (R)a[3 * i + 2]};             \
    });                                                                           \
  }
ORC_SET3(set_velocities, vel)
ORC_SET3(set_external_forces, extForce)
ORC_SET3(set_angular_velocities, angVel)
ORC_SET3(set_inv_inertia, invI)
int orc_clear_external_forces(void* h) {
  return with(h, [&](auto& S) {
    for (auto& f : S.extForce)
      f = {0, 0, 0};
  });
}
int orc_set_quaternions(void* h, const double* q, int n) {
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    for (int i = 0; i < S.numReal && i < n; ++i)
      S.quat[i] = {(R)q[4 * i], (R)q[4 * i + 1], (R)q[4 * i + 2], (R)q[4 * i + 3]};
  });
}
int orc_set_inv_mass(void* h, const double* a, int n) {
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    for (int i = 0; i < S.numReal && i < n; ++i)
      S.invMass[i] = (R)a[i];
  });
}
int orc_set_scales(void* h, const double* a, int n) {  // sim.hpp:1340-1346
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    for (int i = 0; i < S.numReal && i < n; ++i)
      S.targetScale[i] = (R)a[i];
    S.scale = S.targetScale;
  });
}
int orc_set_scales_uniform(void* h, double s) {  // sim.hpp:1331-1337
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    for (int i = 0; i < S.numReal; ++i)
      S.scale[i] = (R)s;
    S.targetScale = S.scale;
  });
}
int orc_set_growth_params(void* h, double rate, double nf) {  // sim.hpp:1416-1424
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    const R r = (R)rate, f = (R)nf;
    if (S.growthFactor == R(-1))
      S.growthFactor = (f > R(0)) ? f : R(0.01);
    else if (f > R(0))
      S.growthFactor = f;
    S.growthRate = r;
    if (S.growthFactor > R(0))
      S.updateGrowthScales(S.numReal, S.growthFactor);
  });
}
double orc_get_growth_factor(void* h) {
  double v = 0;
  with(h, [&](auto& S) { v = dv(S.growthFactor); });
  return v;
}
double orc_get_growth_rate(void* h) {
  double v = 0;
  with(h, [&](auto& S) { v = dv(S.growthRate); });
  return v;
}
#define ORC_GET3(NAME, FIELD)                                          \
  long orc_##NAME(void* h, double* out, long cap) {                    \
    long n = 0;                                                        \
    with(h, [&](auto& S) {                                             \
      n = 3L * S.numReal;                                              \
      for (long i = 0; i < S.numReal && 3 * i + 2 < cap; ++i) {        \
        out[3 * i] = dv(S.FIELD[i].x);                                     \
        out[3 * i + 1] = dv(S.FIELD[i].y);                                 \
        out[3 * i + 2] = dv(S.FIELD[i].z);                                 \
      }                                                                \
    });                                                                \
    return n;                                                          \
  }
ORC_GET3(get_positions, pos)
ORC_GET3(get_velocities, vel)
ORC_GET3(get_angular_velocities, angVel)
ORC_GET3(get_inv_inertia, invI)
long orc_get_quaternions(void* h, double* out, long cap) {
  long n = 0;
  with(h, [&](auto& S) {
    n = 4L * S.numReal;
    for (long i = 0; i < S.numReal && 4 * i + 3 < cap; ++i) {
      out[4 * i] = dv(S.quat[i].x);
      out[4 * i + 1] = dv(S.quat[i].y);
      out[4 * i + 2] = dv(S.quat[i].z);
      out[4 * i + 3] = dv(S.quat[i].w);
    }
  });
  return n;
}
long orc_get_scales(void* h, double* out, long cap) {
  long n = 0;
  with(h, [&](auto& S) {
    n = S.numReal;
    for (long i = 0; i < n && i < cap; ++i)
      out[i] = dv(S.scale[i]);
  });
  return n;
}
long orc_get_masses(void* h, double* out, long cap) {
  long n = 0;
  with(h, [&](auto& S) {
    using R = decltype(S.dt);
    n = S.numReal;
    for (long i = 0; i < n && i < cap; ++i)
      out[i] = (S.invMass[i] > R(0)) ? (double)(R(1) / S.invMass[i]) : 0.0;
  });
  return n;
}
int orc_step(void* h, double dt) {
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    S.dt = (R)dt;
    S.demStep();
  });
}
int orc_step_hertz(void* h, double dt, int substeps, double skin) {
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    S.stepHertz((R)dt, substeps, (R)skin);
  });
}
int orc_compute_overlaps(void* h, double* out) {
  return with(h, [&](auto& S) { *out = dv(S.computeOverlaps()); });
}
int orc_num_particles(void* h) {
  int n = 0;
  with(h, [&](auto& S) { n = S.numReal; });
  return n;
}
int orc_num_contacts(void* h) {
  int n = 0;
  with(h, [&](auto& S) { n = S.contactCount; });
  return n;
}
int orc_num_manifolds(void* h) {
  int n = 0;
  with(h, [&](auto& S) { n = S.manifoldCount; });
  return n;
}
double orc_max_overlap(void* h) {
  double v = 0;
  with(h, [&](auto& S) { v = dv(S.maxOverlap); });
  return v;
}
int orc_get_domain(void* h, double* mn, double* mx) {
  return with(h, [&](auto& S) {
    mn[0] = dv(S.dmin.x), mn[1] = dv(S.dmin.y), mn[2] = dv(S.dmin.z);
    mx[0] = dv(S.dmax.x), mx[1] = dv(S.dmax.y), mx[2] = dv(S.dmax.z);
  });
}
long orc_get_sdf_grid(void* h, int rx, int ry, int rz, double* out, long cap) {
  long n = -1;
  const int st = with(h, [&](auto& S) {
    if (rx < 1 || ry < 1 || rz < 1)
      throw std::invalid_argument("get_sdf_grid: resolution must be positive");
    const auto g = S.generateSdf(rx, ry, rz);
    n = (long)g.size();
    for (long i = 0; i < n && i < cap; ++i)
      out[i] = (double)g[i];
  });
  return st == 0 ? n : -1;
}
int orc_export_lammps(void*, const char*, int) {
  g_err = "oracle: export not restated";
  return 3;
}
int orc_write_vtp(void*, const char*) {
  g_err = "oracle: export not restated";
  return 3;
}

// ---- diagnostics (same layouts as the B200 library) ----
int orc_debug_counts(void* h, long* out) {
  return with(h, [&](auto& S) {
    out[0] = S.pairCount;
    out[1] = S.contactCount;
    out[2] = S.manifoldCount;
    out[3] = S.numParticles;
    out[4] = S.prevPairCount;
    out[5] = S.capacity;
    out[6] = S.maxContacts;
    out[7] = S.maxPairs;
  });
}
long orc_debug_pairs(void* h, int* out, long cap) {
  long n = 0;
  with(h, [&](auto& S) {
    n = std::min(S.pairCount, S.maxPairs);
    for (long i = 0; i < n && 2 * i + 1 < cap; ++i) {
      out[2 * i] = S.pairs[2 * i];
      out[2 * i + 1] = S.pairs[2 * i + 1];
    }
  });
  return n;
}
long orc_debug_contacts(void* h, double* out, long cap) {
  long n = 0;
  with(h, [&](auto& S) {
    n = S.contactCount;
    for (long i = 0; i < n && 17 * i + 16 < cap; ++i) {
      const auto& c = S.contacts[i];
      const double v[17] = {(double)c.a, (double)c.b, dv(c.n.x), dv(c.n.y), dv(c.n.z), dv(c.rA.x), dv(c.rA.y), dv(c.rA.z),
                            dv(c.rB.x), dv(c.rB.y), dv(c.rB.z), dv(c.dist), dv(c.lamN), dv(c.bvel.x), dv(c.bvel.y), dv(c.bvel.z), dv(c.e)};
      std::memcpy(out + 17 * i, v, sizeof v);
    }
  });
  return n;
}
long orc_debug_contact_mu(void* h, double* out, long cap) {
  long n = 0;
  with(h, [&](auto& S) {
    n = S.contactCount;
    for (long i = 0; i < n && i < cap; ++i)
      out[i] = dv(S.contacts[i].mu);
  });
  return n;
}
long orc_debug_manifolds(void* h, double* out, long cap) {
  long n = 0;
  with(h, [&](auto& S) {
    n = S.manifoldCount;
    for (long i = 0; i < n && 23 * i + 22 < cap; ++i) {
      const auto& m = S.manifolds[i];
      const double v[23] = {(double)m.a, (double)m.b, dv(m.N.x),  dv(m.N.y),  dv(m.N.z),  dv(m.TA.x),
                            dv(m.TA.y),      dv(m.TA.z),      dv(m.TB.x), dv(m.TB.y), dv(m.TB.z), dv(m.rA.x),
                            dv(m.rA.y),      dv(m.rA.z),      dv(m.rB.x), dv(m.rB.y), dv(m.rB.z), (double)m.np,
                            dv(m.wv.x),      dv(m.wv.y),      dv(m.wv.z), dv(m.e),    dv(m.mu)};
      std::memcpy(out + 23 * i, v, sizeof v);
    }
  });
  return n;
}
long orc_debug_manifold_colors(void* h, int* out, long cap) {
  long n = 0;
  with(h, [&](auto& S) {
    n = S.manifoldCount;
    for (long i = 0; i < n && i < cap; ++i)
      out[i] = S.mColor[i];
  });
  return n;
}
long orc_debug_contact_colors(void* h, int* out, long cap) {
  long n = 0;
  with(h, [&](auto& S) {
    n = S.contactCount;
    for (long i = 0; i < n && i < cap; ++i)
      out[i] = S.cColor[i];
  });
  return n;
}
long orc_debug_lambda(void* h, double* out, long cap) {
  long n = 0;
  with(h, [&](auto& S) {
    n = S.manifoldCount;
    for (long i = 0; i < n && 4 * i + 3 < cap; ++i) {
      out[4 * i] = dv(S.lambdaAcc[i]);
      out[4 * i + 1] = dv(S.lambdaT[i].x);
      out[4 * i + 2] = dv(S.lambdaT[i].y);
      out[4 * i + 3] = dv(S.lambdaT[i].z);
    }
  });
  return n;
}
long orc_debug_pair_keys(void* h, unsigned long long* out, long cap) {
  long n = 0;
  with(h, [&](auto& S) {
    n = S.manifoldCount;
    for (long i = 0; i < n && i < cap; ++i)
      out[i] = S.pairKeys[i];
  });
  return n;
}
long orc_debug_ledger(void* h, unsigned long long* keys, double* vals, long cap) {
  long n = 0;
  with(h, [&](auto& S) {
    n = S.prevPairCount;
    for (long i = 0; i < n && i < cap; ++i) {
      keys[i] = S.prevPairKeys[i];
      vals[5 * i] = dv(S.prevLambda[i]);
      vals[5 * i + 1] = dv(S.prevLambdaT[i].x);
      vals[5 * i + 2] = dv(S.prevLambdaT[i].y);
      vals[5 * i + 3] = dv(S.prevLambdaT[i].z);
      vals[5 * i + 4] = dv(S.prevPosImpulse[i]);
    }
  });
  return n;
}
long orc_debug_grounded(void* h, int* out, long cap) {
  long n = 0;
  with(h, [&](auto& S) {
    n = S.numReal;
    for (long i = 0; i < n && i < cap; ++i)
      out[i] = S.grounded[i];
  });
  return n;
}
long orc_debug_pos_lambda(void* h, double* out, long cap) {
  long n = 0;
  with(h, [&](auto& S) {
    n = S.contactCount;
    for (long i = 0; i < n && i < cap; ++i)
      out[i] = dv(S.posLambdaContact[i]);
  });
  return n;
}
long orc_debug_hertz(void* h, unsigned long long* keys, double* xi, long cap) {
  long n = 0;
  with(h, [&](auto& S) {
    n = S.hzNumPairs;
    for (long i = 0; i < n && i < cap; ++i) {
      keys[i] = S.hzKeys[i];
      xi[3 * i] = dv(S.hzXi[i].x);
      xi[3 * i + 1] = dv(S.hzXi[i].y);
      xi[3 * i + 2] = dv(S.hzXi[i].z);
    }
  });
  return n;
}
int orc_debug_set_max_contacts(void* h, int maxC) {
  return with(h, [&](auto& S) {
    using R = decltype(S.dt);
    S.contacts.assign(maxC, orc::Contact<R>{});
    S.maxContacts = maxC;
  });
}

// Tangent lanes of the dual-number oracle (precision 65). `which`: 0 positions, 1 velocities,
// 2 angular velocities (n x 3 each), 3 quaternions (n x 4), 4 the material (eN, eT, mu). Seeding
// sets lane `lane` of those values to t; reading returns it. Status 2 when the handle is not dual.
}  // extern "C"
namespace {
template <class F>
int dualDo(void* h, F&& fn) {
  Handle* H = static_cast<Handle*>(h);
  if (!H->x) {
    g_err = "not a dual-number oracle (precision 65)";
    return 2;
  }
  fn(*H->x);
  return 0;
}
template <class G>
void dualFields(orc::Sim<orc::Dual>& S, int which, long n, G&& g) {
  if (which >= 0 && which <= 2) {
    auto& f = which == 0 ? S.pos : which == 1 ? S.vel : S.angVel;
    for (long i = 0; i < n; ++i) {
      g(f[i].x, 3 * i);
      g(f[i].y, 3 * i + 1);
      g(f[i].z, 3 * i + 2);
    }
  } else if (which == 3) {
    for (long i = 0; i < n; ++i) {
      g(S.quat[i].x, 4 * i);
      g(S.quat[i].y, 4 * i + 1);
      g(S.quat[i].z, 4 * i + 2);
      g(S.quat[i].w, 4 * i + 3);
    }
  } else if (which == 4) {
    g(S.eN, 0);
    g(S.eT, 1);
    g(S.mu, 2);
  }
}
}  // namespace
extern "C" {

int orc_dual_seed(void* h, int which, int lane, const double* t, long n) {
  if (lane < 0 || lane >= orc::kDualLanes || which < 0 || which > 4)
    return 2;
  return dualDo(h, [&](orc::Sim<orc::Dual>& S) {
    dualFields(S, which, std::min<long>(n, S.numReal), [&](orc::Dual& x, long k) { x.d[lane] = t[k]; });
  });
}
int orc_dual_get(void* h, int which, int lane, double* t, long n) {
  if (lane < 0 || lane >= orc::kDualLanes || which < 0 || which > 4)
    return 2;
  return dualDo(h, [&](orc::Sim<orc::Dual>& S) {
    dualFields(S, which, std::min<long>(n, S.numReal), [&](orc::Dual& x, long k) { t[k] = x.d[lane]; });
  });
}
int orc_dual_lanes() { return orc::kDualLanes; }

}  // extern "C"
