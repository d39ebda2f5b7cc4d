// C API over the UNMODIFIED reference peclet::dem::Simulation (test infrastructure).
//
// Compiled by oracle/Makefile against the Kokkos/ArborX shim (oracle/kokkos_shim) from the reference
// headers where they lie (REF_SRC/src), into oracle/_ref/. The exported `ref_*` functions mirror the
// reference binding (src/dem_bindings.cpp:72-464) one to one, with double-precision host arrays at
// the boundary (converted to the reference's float), plus read-only debug getters for the step's
// intermediate products (candidate pairs, contacts, manifolds, colours, warm-start ledger) so the
// parity tests can compare them bit for bit. The Simulation's private Particles SoA is reached by
// compiling the header with `private` mapped to `public` in this translation unit only.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <fstream>
#include <iomanip>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include <ArborX.hpp>
#include <Kokkos_Core.hpp>
#include <Kokkos_Sort.hpp>
#include <peclet/core/common/view.hpp>

#define private public
#include "sim.hpp"
#undef private

using peclet::dem::F3;
using peclet::dem::Simulation;

namespace {
thread_local std::string g_err;
template <class F>
int guard(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::invalid_argument& e) {
    g_err = e.what();
    return 2;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}
std::vector<float> tof(const double* p, long n) {
  std::vector<float> v(n > 0 ? n : 0);
  for (long i = 0; i < n; ++i)
    v[i] = static_cast<float>(p[i]);
  return v;
}
Simulation* S(void* h) { return static_cast<Simulation*>(h); }
long copyOut(const std::vector<float>& v, double* out, long cap) {
  const long n = static_cast<long>(v.size());
  for (long i = 0; i < n && i < cap; ++i)
    out[i] = v[i];
  return n;
}
}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }
const char* ref_execution_space() { return Kokkos::DefaultExecutionSpace::name(); }

// `precision` is accepted for signature parity with the other implementations; the reference
// computes in float only.
int ref_create(int capacity, int precision, void** out) {
  (void)precision;
  if (!Kokkos::is_initialized())
    Kokkos::initialize();
  return guard([&] { *out = new Simulation(capacity); });
}
void ref_destroy(void* h) { delete S(h); }

int ref_initialize_shape(void* h, int type, double r, double height, double thick) {
  return guard([&] { S(h)->initializeShape(type, (float)r, (float)height, (float)thick); });
}
int ref_set_sdf_shape(void* h, const double* grid, int nx, int ny, int nz, const double* origin,
                      const double* spacing, const double* shell, int nshell,
                      const double* invI, double boundingRadius) {
  return guard([&] {
    S(h)->setSdfShape(tof(grid, (long)nx * ny * nz), nx, ny, nz,
                      F3{(float)origin[0], (float)origin[1], (float)origin[2]},
                      F3{(float)spacing[0], (float)spacing[1], (float)spacing[2]},
                      tof(shell, (long)nshell * 3), F3{(float)invI[0], (float)invI[1], (float)invI[2]},
                      (float)boundingRadius);
  });
}
int ref_set_shell_points(void* h, const double* pts, int n) {
  // Replace shape 0's analytic point shell (the shape's SDF stays analytic). Sets the Particles
  // shell and ShapeDesc.numPoints directly, as the facade has no setter for it.
  return guard([&] {
    auto& P = S(h)->P_;
    P.shell = Kokkos::View<float* [3], peclet::dem::CpMem>("shell", n > 0 ? n : 1);
    for (int i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d)
        P.shell(i, d) = (float)pts[3 * i + d];
    P.shapes(0).numPoints = n;
    P.shapes(0).shellOffset = 0;
    S(h)->shellPoints_ = n;
    S(h)->ensureContactCapacity();
  });
}
int ref_set_domain(void* h, double lx, double ly, double lz, int px, int py, int pz) {
  return guard([&] { S(h)->setDomain((float)lx, (float)ly, (float)lz, px, py, pz); });
}
int ref_set_domain_minmax(void* h, const double* mn, const double* mx) {
  return guard([&] {
    S(h)->setDomainMinMax(F3{(float)mn[0], (float)mn[1], (float)mn[2]},
                          F3{(float)mx[0], (float)mx[1], (float)mx[2]});
  });
}
int ref_enable_periodicity(void* h, int x, int y, int z) {
  return guard([&] { S(h)->enablePeriodicity(x, y, z); });
}
int ref_set_gravity(void* h, double gx, double gy, double gz) {
  return guard([&] { S(h)->setGravity((float)gx, (float)gy, (float)gz); });
}
int ref_set_thermostat(void* h, double T, double tau, double kB) {
  return guard([&] { S(h)->setThermostat((float)T, (float)tau, (float)kB); });
}
int ref_set_solver_iterations(void* h, int pos, int vel) {
  return guard([&] { S(h)->setSolverIterations(pos, vel); });
}
int ref_set_velocity_use_gs(void* h, int b) {
  return guard([&] { S(h)->setVelocityUseGS(b != 0); });
}
int ref_set_stabilization_mode(void* h, const char* mode) {
  return guard([&] { S(h)->setStabilizationMode(mode); });
}
int ref_set_hertz_material(void* h, int mat, double E, double nu) {
  return guard([&] { S(h)->setHertzMaterial(mat, (float)E, (float)nu); });
}
int ref_set_global_scale(void* h, double s) { return guard([&] { S(h)->setGlobalScale((float)s); }); }
int ref_set_dt(void* h, double dt) { return guard([&] { S(h)->setDt((float)dt); }); }
int ref_set_material_params(void* h, double en, double et, double mu) {
  return guard([&] { S(h)->setMaterialParams((float)en, (float)et, (float)mu); });
}
int ref_set_material_ids(void* h, const int* ids, int n) {
  return guard([&] { S(h)->setMaterialIds(std::vector<int>(ids, ids + n)); });
}
int ref_set_pair_material(void* h, int a, int b, double e, double mu) {
  return guard([&] { S(h)->setPairMaterial(a, b, (float)e, (float)mu); });
}
int ref_set_wall_material_id(void* h, int wid, int mat) {
  return guard([&] { S(h)->setWallMaterialId(wid, mat); });
}
int ref_add_plane(void* h, double px, double py, double pz, double nx, double ny, double nz) {
  return guard([&] {
    S(h)->addPlane((float)px, (float)py, (float)pz, (float)nx, (float)ny, (float)nz);
  });
}
int ref_add_sdf_wall(void* h, const double* grid, int nx, int ny, int nz, const double* origin,
                     const double* spacing, double e, double mu, int* outIdx) {
  return guard([&] {
    *outIdx = S(h)->addSdfWall(tof(grid, (long)nx * ny * nz), nx, ny, nz,
                               F3{(float)origin[0], (float)origin[1], (float)origin[2]},
                               F3{(float)spacing[0], (float)spacing[1], (float)spacing[2]},
                               (float)e, (float)mu);
  });
}
int ref_set_wall_velocity(void* h, int idx, const double* lin, const double* ang,
                          const double* center) {
  return guard([&] {
    S(h)->setWallVelocity(idx, F3{(float)lin[0], (float)lin[1], (float)lin[2]},
                          F3{(float)ang[0], (float)ang[1], (float)ang[2]},
                          F3{(float)center[0], (float)center[1], (float)center[2]});
  });
}
int ref_set_positions(void* h, const double* xyz, int n) {
  return guard([&] { S(h)->setPositions(tof(xyz, (long)n * 3)); });
}
int ref_set_velocities(void* h, const double* v, int n) {
  return guard([&] { S(h)->setVelocities(tof(v, (long)n * 3)); });
}
int ref_set_external_forces(void* h, const double* f, int n) {
  return guard([&] { S(h)->setExternalForces(tof(f, (long)n * 3)); });
}
int ref_clear_external_forces(void* h) { return guard([&] { S(h)->clearExternalForces(); }); }
int ref_set_quaternions(void* h, const double* q, int n) {
  return guard([&] { S(h)->setQuaternions(tof(q, (long)n * 4)); });
}
int ref_set_angular_velocities(void* h, const double* w, int n) {
  return guard([&] { S(h)->setAngularVelocities(tof(w, (long)n * 3)); });
}
int ref_set_inv_inertia(void* h, const double* ii, int n) {
  return guard([&] { S(h)->setInvInertia(tof(ii, (long)n * 3)); });
}
int ref_set_inv_mass(void* h, const double* im, int n) {
  return guard([&] { S(h)->setInvMass(tof(im, n)); });
}
int ref_set_scales(void* h, const double* s, int n) {
  return guard([&] { S(h)->setScales(tof(s, n)); });
}
int ref_set_scales_uniform(void* h, double s) {
  return guard([&] { S(h)->setScalesUniform((float)s); });
}
int ref_set_growth_params(void* h, double rate, double nf) {
  return guard([&] { S(h)->setGrowthParams((float)rate, (float)nf); });
}
double ref_get_growth_factor(void* h) { return S(h)->growthFactor(); }
double ref_get_growth_rate(void* h) { return S(h)->getGrowthRate(); }

long ref_get_positions(void* h, double* out, long cap) {
  return copyOut(S(h)->getPositions(), out, cap);
}
long ref_get_velocities(void* h, double* out, long cap) {
  return copyOut(S(h)->getVelocities(), out, cap);
}
long ref_get_quaternions(void* h, double* out, long cap) {
  return copyOut(S(h)->getQuaternions(), out, cap);
}
long ref_get_angular_velocities(void* h, double* out, long cap) {
  return copyOut(S(h)->getAngularVelocities(), out, cap);
}
long ref_get_inv_inertia(void* h, double* out, long cap) {
  return copyOut(S(h)->getInvInertia(), out, cap);
}
long ref_get_scales(void* h, double* out, long cap) { return copyOut(S(h)->getScales(), out, cap); }
long ref_get_masses(void* h, double* out, long cap) { return copyOut(S(h)->getMasses(), out, cap); }

int ref_step(void* h, double dt) { return guard([&] { S(h)->step((float)dt); }); }
int ref_step_hertz(void* h, double dt, int substeps, double skin) {
  return guard([&] { S(h)->stepHertz((float)dt, substeps, (float)skin); });
}
int ref_compute_overlaps(void* h, double* out) {
  return guard([&] { *out = S(h)->computeOverlaps(); });
}
int ref_num_particles(void* h) { return S(h)->numParticles(); }
int ref_num_contacts(void* h) { return S(h)->numContacts(); }
int ref_num_manifolds(void* h) { return S(h)->numManifolds(); }
double ref_max_overlap(void* h) { return S(h)->maxOverlap(); }
int ref_export_lammps(void* h, const char* fn, int step) {
  return guard([&] { S(h)->exportLammps(fn, step); });
}
int ref_write_vtp(void* h, const char* fn) { return guard([&] { S(h)->writeVtp(fn); }); }
int ref_get_domain(void* h, double* mn, double* mx) {
  return guard([&] {
    const auto a = S(h)->getDomainMin();
    const auto b = S(h)->getDomainMax();
    mn[0] = std::get<0>(a), mn[1] = std::get<1>(a), mn[2] = std::get<2>(a);
    mx[0] = std::get<0>(b), mx[1] = std::get<1>(b), mx[2] = std::get<2>(b);
  });
}
long ref_get_sdf_grid(void* h, int rx, int ry, int rz, double* out, long cap) {
  long n = -1;
  const int st = guard([&] { n = copyOut(S(h)->getSdfGrid(rx, ry, rz), out, cap); });
  return st == 0 ? n : -1;
}
int ref_export_sdf(void* h, const char* fn, int rx, int ry, int rz) {
  return guard([&] { S(h)->exportSdf(fn, rx, ry, rz); });
}

// ---- debug getters: the step's intermediate products ----
int ref_debug_counts(void* h, long* out) {
  auto& P = S(h)->P_;
  out[0] = P.pairCount();
  out[1] = P.contactCount();
  out[2] = P.manifoldCount();
  out[3] = P.numParticles;
  out[4] = P.prevPairCount;
  out[5] = P.capacity;
  out[6] = P.maxContacts;
  out[7] = (long)P.pairs.extent(0);
  return 0;
}
long ref_debug_pairs(void* h, int* out, long cap) {
  auto& P = S(h)->P_;
  const long n = std::min<long>(P.pairCount(), (long)P.pairs.extent(0));
  for (long i = 0; i < n && 2 * i + 1 < cap; ++i) {
    out[2 * i] = P.pairs(i, 0);
    out[2 * i + 1] = P.pairs(i, 1);
  }
  return n;
}
// 17 doubles per contact: bodyA bodyB n(3) rA(3) rB(3) dist lambdaN bvel(3) e mu
long ref_debug_contacts(void* h, double* out, long cap) {
  auto& P = S(h)->P_;
  const long n = P.contactCount();
  for (long i = 0; i < n && 17 * i + 16 < cap; ++i) {
    const auto& c = P.contacts(i);
    double* o = out + 17 * i;
    o[0] = c.bodyA;
    o[1] = c.bodyB;
    o[2] = c.normal.x;
    o[3] = c.normal.y;
    o[4] = c.normal.z;
    o[5] = c.rA.x;
    o[6] = c.rA.y;
    o[7] = c.rA.z;
    o[8] = c.rB.x;
    o[9] = c.rB.y;
    o[10] = c.rB.z;
    o[11] = c.dist;
    o[12] = c.friction_lambda_n;
    o[13] = c.boundaryVel.x;
    o[14] = c.boundaryVel.y;
    o[15] = c.boundaryVel.z;
    o[16] = c.boundaryRestitution;
    (void)0;
  }
  return n;
}
long ref_debug_contact_mu(void* h, double* out, long cap) {
  auto& P = S(h)->P_;
  const long n = P.contactCount();
  for (long i = 0; i < n && i < cap; ++i)
    out[i] = P.contacts(i).boundaryFriction;
  return n;
}
// 23 doubles per manifold: bodyA bodyB Nsum(3) TauA(3) TauB(3) rA(3) rB(3) npts wvel(3) e mu
long ref_debug_manifolds(void* h, double* out, long cap) {
  auto& P = S(h)->P_;
  const long n = P.manifoldCount();
  for (long i = 0; i < n && 23 * i + 22 < cap; ++i) {
    const auto& m = P.manifolds(i);
    double* o = out + 23 * i;
    o[0] = m.bodyA;
    o[1] = m.bodyB;
    o[2] = m.normal_sum.x;
    o[3] = m.normal_sum.y;
    o[4] = m.normal_sum.z;
    o[5] = m.torque_armA_sum.x;
    o[6] = m.torque_armA_sum.y;
    o[7] = m.torque_armA_sum.z;
    o[8] = m.torque_armB_sum.x;
    o[9] = m.torque_armB_sum.y;
    o[10] = m.torque_armB_sum.z;
    o[11] = m.rA_sum.x;
    o[12] = m.rA_sum.y;
    o[13] = m.rA_sum.z;
    o[14] = m.rB_sum.x;
    o[15] = m.rB_sum.y;
    o[16] = m.rB_sum.z;
    o[17] = m.num_points;
    o[18] = m.wallVel_sum.x;
    o[19] = m.wallVel_sum.y;
    o[20] = m.wallVel_sum.z;
    o[21] = m.restitution_sum;
    o[22] = m.friction_sum;
  }
  return n;
}
long ref_debug_manifold_colors(void* h, int* out, long cap) {
  auto& P = S(h)->P_;
  const long n = P.manifoldCount();
  for (long i = 0; i < n && i < cap; ++i)
    out[i] = P.manifoldColor(i);
  return n;
}
long ref_debug_contact_colors(void* h, int* out, long cap) {
  auto& P = S(h)->P_;
  const long n = P.contactCount();
  for (long i = 0; i < n && i < cap; ++i)
    out[i] = P.contactColor(i);
  return n;
}
// per manifold: lambdaAcc, lambdaT(3), pairKey (as double bits via separate getter)
long ref_debug_lambda(void* h, double* out, long cap) {
  auto& P = S(h)->P_;
  const long n = P.manifoldCount();
  for (long i = 0; i < n && 4 * i + 3 < cap; ++i) {
    out[4 * i] = P.lambdaAcc(i);
    out[4 * i + 1] = P.lambdaT(i, 0);
    out[4 * i + 2] = P.lambdaT(i, 1);
    out[4 * i + 3] = P.lambdaT(i, 2);
  }
  return n;
}
long ref_debug_pair_keys(void* h, unsigned long long* out, long cap) {
  auto& P = S(h)->P_;
  const long n = P.manifoldCount();
  for (long i = 0; i < n && i < cap; ++i)
    out[i] = P.pairKeys(i);
  return n;
}
// committed ledger (sorted): prevPairKeys, prevLambda, prevLambdaT(3), prevPosImpulse
long ref_debug_ledger(void* h, unsigned long long* keys, double* vals, long cap) {
  auto& P = S(h)->P_;
  const long n = P.prevPairCount;
  for (long i = 0; i < n && i < cap; ++i) {
    keys[i] = P.prevPairKeys(i);
    vals[5 * i] = P.prevLambda(i);
    vals[5 * i + 1] = P.prevLambdaT(i, 0);
    vals[5 * i + 2] = P.prevLambdaT(i, 1);
    vals[5 * i + 3] = P.prevLambdaT(i, 2);
    vals[5 * i + 4] = P.prevPosImpulse(i);
  }
  return n;
}
long ref_debug_grounded(void* h, int* out, long cap) {
  auto& P = S(h)->P_;
  const long n = P.numReal;
  for (long i = 0; i < n && i < cap; ++i)
    out[i] = P.groundedLevel(i);
  return n;
}
long ref_debug_pos_lambda(void* h, double* out, long cap) {
  auto& P = S(h)->P_;
  const long n = P.contactCount();
  for (long i = 0; i < n && i < cap; ++i)
    out[i] = P.posLambdaContact(i);
  return n;
}
// Hertz cached list: pairs count, keys, xi(3)
long ref_debug_hertz(void* h, unsigned long long* keys, double* xi, long cap) {
  auto& P = S(h)->P_;
  const long n = P.hertzNumPairs;
  for (long i = 0; i < n && i < cap; ++i) {
    keys[i] = P.hertzKeys(i);
    xi[3 * i] = P.hertzXi(i, 0);
    xi[3 * i + 1] = P.hertzXi(i, 1);
    xi[3 * i + 2] = P.hertzXi(i, 2);
  }
  return n;
}
// Test hook: shrink the contact buffers (overflow/clamp behaviour tests).
int ref_debug_set_max_contacts(void* h, int maxC) {
  auto& P = S(h)->P_;
  P.contacts = Kokkos::View<peclet::dem::ContactC*, peclet::dem::CpMem>("contacts", maxC);
  P.maxContacts = maxC;
  return 0;
}

}  // extern "C"
