// C ABI of the B200 substep (declared in include/pdem.h). Thin: each entry point converts host
// arrays to the handle's precision, calls the Sim<R> facade and maps exceptions to status codes.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <limits>
#include <string>
#include <vector>

#include "../../include/pdem.h"
#include "pdem_radix.cuh"
#include "pdem_sim.cuh"
#include "pdem_xadj_api.cuh"

using pdem::Sim;

namespace {
thread_local std::string g_err;
std::string g_space;

struct Handle {
  Sim<float>* f = nullptr;
  Sim<double>* d = nullptr;
};

template <class F>
int with(pdem_handle h, F&& fn) {
  if (!h) {
    g_err = "null simulation handle";
    return PDEM_ERR_INVALID;
  }
  Handle* H = static_cast<Handle*>(h);
  // a read-back queued before an exception must not be delivered to a dead frame by a later sync
  auto drop = [&] { H->f ? H->f->dropPending() : H->d->dropPending(); };
  try {
    if (H->f)
      fn(*H->f);
    else
      fn(*H->d);
    return PDEM_OK;
  } catch (const std::invalid_argument& e) {
    drop();
    g_err = e.what();
    return PDEM_ERR_INVALID;
  } catch (const pdem::CudaError& e) {
    drop();
    g_err = e.what();
    return PDEM_ERR_CUDA;
  } catch (const std::exception& e) {
    drop();
    g_err = e.what();
    return PDEM_ERR_RUNTIME;
  }
}
template <class R>
std::vector<R> conv(const double* p, long n) {
  std::vector<R> v(n > 0 ? n : 0);
  for (long i = 0; i < n; ++i)
    v[i] = static_cast<R>(p[i]);
  return v;
}
template <class S>
using RealOf = std::remove_reference_t<decltype(std::declval<S&>().dt_)>;

// LAMMPS "dump custom" writer, format of src/io.hpp:23-82 (id type x y z radius vx vy vz qw qx qy qz)
void writeLammps(const std::string& fn, int step, const std::vector<double>& pos, const std::vector<double>& vel,
                 const std::vector<double>& quat, const std::vector<double>& radii, bool pbc) {
  const size_t n = pos.size() / 3;
  float lo[3], hi[3];
  if (n == 0) {
    for (int a = 0; a < 3; ++a)
      lo[a] = hi[a] = 0.0f;
  } else {
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::numeric_limits<float>::max();
      hi[a] = -std::numeric_limits<float>::max();
    }
    for (size_t i = 0; i < n; ++i)
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], (float)pos[3 * i + a] - (float)radii[i]);
        hi[a] = std::max(hi[a], (float)pos[3 * i + a] + (float)radii[i]);
      }
    for (int a = 0; a < 3; ++a) {
      const float m = 0.05f * (hi[a] - lo[a]);
      lo[a] -= m;
      hi[a] += m;
    }
  }
  std::ofstream f(fn);
  if (!f)
    throw std::runtime_error("Could not open file for writing: " + fn);
  f << "ITEM: TIMESTEP\n" << step << "\n";
  f << "ITEM: NUMBER OF ATOMS\n" << n << "\n";
  f << "ITEM: BOX BOUNDS " << (pbc ? "pp pp pp" : "ff ff ff") << "\n";
  for (int a = 0; a < 3; ++a)
    f << lo[a] << " " << hi[a] << "\n";
  f << "ITEM: ATOMS id type x y z radius vx vy vz qw qx qy qz\n";
  f << std::fixed << std::setprecision(6);
  for (size_t i = 0; i < n; ++i)
    f << (i + 1) << " 1 " << pos[3 * i] << " " << pos[3 * i + 1] << " " << pos[3 * i + 2] << " " << radii[i] << " "
      << vel[3 * i] << " " << vel[3 * i + 1] << " " << vel[3 * i + 2] << " " << quat[4 * i + 3] << " "
      << quat[4 * i] << " " << quat[4 * i + 1] << " " << quat[4 * i + 2] << "\n";
}
// ParaView PolyData writer, format of src/sim.hpp:1560-1601 (points + Radius + Velocity)
// ImageData VTI of an SDF grid (src/io.hpp:86-110): ASCII Float32 values in the stream's default
// format, origin at the domain minimum, spacing (max - min) / (res - 1) per axis
template <class T>
void writeSdfVti(const std::string& fn, const std::vector<T>& grid, int rx, int ry, int rz, const float* mn,
                 const float* mx) {
  const double sx = rx > 1 ? (double(mx[0]) - mn[0]) / (rx - 1) : 1.0;
  const double sy = ry > 1 ? (double(mx[1]) - mn[1]) / (ry - 1) : 1.0;
  const double sz = rz > 1 ? (double(mx[2]) - mn[2]) / (rz - 1) : 1.0;
  std::ofstream out(fn);
  if (!out)
    throw std::runtime_error("Could not open file for writing: " + fn);
  out << "<?xml version=\"1.0\"?>\n";
  out << "<VTKFile type=\"ImageData\" version=\"0.1\" byte_order=\"LittleEndian\">\n";
  out << "  <ImageData WholeExtent=\"0 " << (rx - 1) << " 0 " << (ry - 1) << " 0 " << (rz - 1) << "\" Origin=\""
      << mn[0] << " " << mn[1] << " " << mn[2] << "\" Spacing=\"" << sx << " " << sy << " " << sz << "\">\n";
  out << "    <Piece Extent=\"0 " << (rx - 1) << " 0 " << (ry - 1) << " 0 " << (rz - 1) << "\">\n";
  out << "      <PointData Scalars=\"sdf\">\n";
  out << "        <DataArray type=\"Float32\" Name=\"sdf\" format=\"ascii\">\n";
  for (const T v : grid)
    out << (float)v << " ";
  out << "\n        </DataArray>\n";
  out << "      </PointData>\n";
  out << "    </Piece>\n";
  out << "  </ImageData>\n";
  out << "</VTKFile>\n";
  std::printf("Exported SDF VTI: %s\n", fn.c_str());
}
void writeVtp(const std::string& fn, const std::vector<double>& pos, const std::vector<double>& vel,
              const std::vector<double>& radii) {
  const size_t n = pos.size() / 3;
  std::ofstream out(fn);
  if (!out)
    throw std::runtime_error("Could not open file for writing: " + fn);
  out << "<?xml version=\"1.0\"?>\n<VTKFile type=\"PolyData\" version=\"0.1\" byte_order=\"LittleEndian\">\n";
  out << "  <PolyData>\n    <Piece NumberOfPoints=\"" << n
      << "\" NumberOfVerts=\"0\" NumberOfLines=\"0\" NumberOfStrips=\"0\" NumberOfPolys=\"0\">\n";
  out << "      <Points>\n        <DataArray type=\"Float32\" Name=\"Position\" NumberOfComponents=\"3\" "
         "format=\"ascii\">\n";
  for (size_t i = 0; i < n; ++i)
    out << pos[3 * i] << " " << pos[3 * i + 1] << " " << pos[3 * i + 2] << " ";
  out << "\n        </DataArray>\n      </Points>\n      <PointData Scalars=\"Radius\">\n";
  out << "        <DataArray type=\"Float32\" Name=\"Radius\" NumberOfComponents=\"1\" format=\"ascii\">\n";
  for (size_t i = 0; i < n; ++i)
    out << radii[i] << " ";
  out << "\n        </DataArray>\n";
  out << "        <DataArray type=\"Float32\" Name=\"Velocity\" NumberOfComponents=\"3\" format=\"ascii\">\n";
  for (size_t i = 0; i < n; ++i)
    out << vel[3 * i] << " " << vel[3 * i + 1] << " " << vel[3 * i + 2] << " ";
  out << "\n        </DataArray>\n      </PointData>\n    </Piece>\n  </PolyData>\n</VTKFile>\n";
  std::printf("Exported VTP: %s\n", fn.c_str());
}
template <class S>
void fetch(S& s, int field, int cols, std::vector<double>& out) {
  using R = RealOf<S>;
  const int n = s.numReal_;
  std::vector<R> h((size_t)n * cols);
  s.getRows(field, h.data(), (long)h.size());
  out.assign(h.begin(), h.end());
}
}  // namespace

namespace pdem {
// message of the last failing entry point, for entry points defined in other translation units
void setLastError(const std::string& msg) { g_err = msg; }
}  // namespace pdem

extern "C" {

const char* pdem_last_error(void) { return g_err.c_str(); }
const char* pdem_execution_space(void) {
  int dev = 0;
  cudaDeviceProp p{};
  if (cudaGetDevice(&dev) == cudaSuccess && cudaGetDeviceProperties(&p, dev) == cudaSuccess)
    g_space = std::string("CUDA sm_100a (") + p.name + ")";
  else
    g_space = "CUDA sm_100a (no device)";
  return g_space.c_str();
}

int pdem_set_device(int device) {
  const cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) {
    g_err = std::string("cudaSetDevice: ") + cudaGetErrorString(e);
    return PDEM_ERR_CUDA;
  }
  return PDEM_OK;
}

int pdem_create(int capacity, int precision, pdem_handle* out) {
  if (!out) {
    g_err = "null output handle";
    return PDEM_ERR_INVALID;
  }
  *out = nullptr;
  if (capacity < 0) {
    g_err = "capacity must be >= 0";
    return PDEM_ERR_INVALID;
  }
  if (precision != 32 && precision != 64 && precision != PDEM_MIXED) {
    g_err = "precision must be 32, 64 or PDEM_MIXED";
    return PDEM_ERR_INVALID;
  }
  int ndev = 0;
  const cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev <= 0) {
    g_err = std::string("no CUDA device available: ") + cudaGetErrorString(e);
    return PDEM_ERR_CUDA;
  }
  Handle* H = new Handle;
  try {
    if (precision == 32 || precision == PDEM_MIXED) {
      H->f = new Sim<float>(capacity);
      H->f->setMixed(precision == PDEM_MIXED);
    } else
      H->d = new Sim<double>(capacity);
  } catch (const std::exception& ex) {
    g_err = ex.what();
    delete H;
    return PDEM_ERR_CUDA;
  }
  *out = H;
  return PDEM_OK;
}
void pdem_destroy(pdem_handle h) {
  if (!h)
    return;
  Handle* H = static_cast<Handle*>(h);
  delete H->f;
  delete H->d;
  delete H;
}

#define BODY(...) return with(h, [&](auto& S) { using R = RealOf<decltype(S)>; (void)sizeof(R); __VA_ARGS__; })

int pdem_initialize_shape(pdem_handle h, int type, double r, double height, double thick) {
  BODY(S.initializeShape(type, (R)r, (R)height, (R)thick));
}
int pdem_set_sdf_shape(pdem_handle h, const double* grid, int nx, int ny, int nz, const double* origin,
                       const double* spacing, const double* shell, int nshell, const double* invI, double bR) {
  BODY({
    const R o[3] = {(R)origin[0], (R)origin[1], (R)origin[2]};
    const R sp[3] = {(R)spacing[0], (R)spacing[1], (R)spacing[2]};
    const R ii[3] = {(R)invI[0], (R)invI[1], (R)invI[2]};
    S.setSdfShape(conv<R>(grid, (long)nx * ny * nz), nx, ny, nz, o, sp, conv<R>(shell, (long)nshell * 3), ii, (R)bR);
  });
}
int pdem_set_shell_points(pdem_handle h, const double* pts, int n) {
  BODY(S.setShellPoints(conv<R>(pts, (long)n * 3)));
}
int pdem_set_domain(pdem_handle h, double lx, double ly, double lz, int px, int py, int pz) {
  BODY(S.setDomain((R)lx, (R)ly, (R)lz, px != 0, py != 0, pz != 0));
}
int pdem_set_domain_minmax(pdem_handle h, const double* mn, const double* mx) {
  BODY({
    const R a[3] = {(R)mn[0], (R)mn[1], (R)mn[2]}, b[3] = {(R)mx[0], (R)mx[1], (R)mx[2]};
    S.setDomainMinMax(a, b);
  });
}
int pdem_enable_periodicity(pdem_handle h, int x, int y, int z) { BODY(S.enablePeriodicity(x, y, z)); }
int pdem_set_gravity(pdem_handle h, double gx, double gy, double gz) { BODY(S.setGravity((R)gx, (R)gy, (R)gz)); }
int pdem_set_thermostat(pdem_handle h, double T, double tau, double kB) {
  BODY(S.setThermostat((R)T, (R)tau, (R)kB));
}
int pdem_set_solver_iterations(pdem_handle h, int pos, int vel) { BODY(S.setSolverIterations(pos, vel)); }
int pdem_set_velocity_use_gs(pdem_handle h, int b) { BODY(S.setVelocityUseGS(b != 0)); }
int pdem_set_stabilization_mode(pdem_handle h, const char* mode) {
  BODY(S.setStabilizationMode(mode ? std::string(mode) : std::string()));
}
int pdem_set_hertz_material(pdem_handle h, int mat, double E, double nu) {
  BODY(S.setHertzMaterial(mat, (R)E, (R)nu));
}
int pdem_set_global_scale(pdem_handle h, double s) { BODY(S.setGlobalScale((R)s)); }
int pdem_set_dt(pdem_handle h, double dt) { BODY(S.setDt((R)dt)); }
int pdem_set_material_params(pdem_handle h, double en, double et, double mu) {
  BODY(S.setMaterialParams((R)en, (R)et, (R)mu));
}
int pdem_set_material_ids(pdem_handle h, const int* ids, int n) { BODY(S.setMaterialIds(ids, n)); }
int pdem_set_pair_material(pdem_handle h, int a, int b, double e, double mu) {
  BODY(S.setPairMaterial(a, b, (R)e, (R)mu));
}
int pdem_set_wall_material_id(pdem_handle h, int wid, int mat) { BODY(S.setWallMaterialId(wid, mat)); }
int pdem_add_plane(pdem_handle h, double px, double py, double pz, double nx, double ny, double nz) {
  BODY({
    const R p[3] = {(R)px, (R)py, (R)pz}, n[3] = {(R)nx, (R)ny, (R)nz};
    S.addPlane(p, n);
  });
}
int pdem_add_sdf_wall(pdem_handle h, const double* grid, int nx, int ny, int nz, const double* origin,
                      const double* spacing, double e, double mu, int* outIdx) {
  BODY({
    const R o[3] = {(R)origin[0], (R)origin[1], (R)origin[2]};
    const R sp[3] = {(R)spacing[0], (R)spacing[1], (R)spacing[2]};
    const int idx = S.addSdfWall(conv<R>(grid, (long)nx * ny * nz), nx, ny, nz, o, sp, (R)e, (R)mu);
    if (outIdx)
      *outIdx = idx;
  });
}
int pdem_set_wall_velocity(pdem_handle h, int idx, const double* lin, const double* ang, const double* c) {
  BODY({
    const R a[3] = {(R)lin[0], (R)lin[1], (R)lin[2]}, b[3] = {(R)ang[0], (R)ang[1], (R)ang[2]},
            cc[3] = {(R)c[0], (R)c[1], (R)c[2]};
    S.setWallVelocity(idx, a, b, cc);
  });
}
int pdem_set_positions(pdem_handle h, const double* xyz, int n) {
  BODY({
    const auto v = conv<R>(xyz, (long)n * 3);
    S.setPositions(v.data(), n);
    S.setMaster(0, xyz, n);
  });
}
#define SETROWS(NAME, FIELD, COLS)                                  \
  int NAME(pdem_handle h, const double* a, int n) {                 \
    BODY({                                                          \
      if (FIELD == 5) {                                             \
        const auto v = conv<R>(a, (long)n * COLS);                  \
        S.setRows(FIELD, v.data(), n);                              \
      } else {                                                      \
        S.setRowsD(FIELD, a, n);                                    \
      }                                                             \
    });                                                             \
  }
SETROWS(pdem_set_velocities, 0, 3)
SETROWS(pdem_set_external_forces, 1, 3)
int pdem_set_quaternions(pdem_handle h, const double* a, int n) {
  BODY({
    S.setRowsD(2, a, n);
    S.setMaster(2, a, n);
  });
}
SETROWS(pdem_set_angular_velocities, 3, 3)
SETROWS(pdem_set_inv_inertia, 4, 3)
SETROWS(pdem_set_inv_mass, 5, 1)
int pdem_clear_external_forces(pdem_handle h) { BODY(S.clearExternalForces()); }
int pdem_set_scales(pdem_handle h, const double* s, int n) {
  BODY({
    const auto v = conv<R>(s, n);
    S.setScales(v.data(), n);
  });
}
int pdem_set_scales_uniform(pdem_handle h, double s) { BODY(S.setScalesUniform((R)s)); }
int pdem_set_growth_params(pdem_handle h, double rate, double nf) { BODY(S.setGrowthParams((R)rate, (R)nf)); }
double pdem_get_growth_factor(pdem_handle h) {
  double v = 0;
  with(h, [&](auto& S) { v = S.growthFactor(); });
  return v;
}
double pdem_get_growth_rate(pdem_handle h) {
  double v = 0;
  with(h, [&](auto& S) { v = S.growthRate(); });
  return v;
}
#define GETROWS(NAME, FIELD, COLS)                                        \
  long NAME(pdem_handle h, double* out, long cap) {                       \
    long n = -1;                                                          \
    with(h, [&](auto& S) {                                                \
      using R = RealOf<decltype(S)>;                                      \
      n = (long)S.numReal_ * COLS;                                        \
      if (S.getMaster(FIELD, out, cap))                                   \
        return;                                                           \
      if (FIELD <= 4) {                                                   \
        S.getRowsD(FIELD, out, cap);                                      \
        return;                                                           \
      }                                                                   \
      std::vector<R> tmp((size_t)std::max(n, 0L));                        \
      S.getRows(FIELD, tmp.data(), (long)tmp.size());                     \
      for (long i = 0; i < n && i < cap; ++i)                             \
        out[i] = tmp[i];                                                  \
    });                                                                   \
    return n;                                                             \
  }
GETROWS(pdem_get_positions, 0, 3)
GETROWS(pdem_get_velocities, 1, 3)
GETROWS(pdem_get_quaternions, 2, 4)
GETROWS(pdem_get_angular_velocities, 3, 3)
GETROWS(pdem_get_inv_inertia, 4, 3)
GETROWS(pdem_get_scales, 5, 1)
GETROWS(pdem_get_masses, 6, 1)

int pdem_step(pdem_handle h, double dt) { BODY(S.step((R)dt)); }
int pdem_step_n(pdem_handle h, double dt, int n) {
  BODY({
    if (n < 0)
      throw std::invalid_argument("step_n: n must be non-negative");
    for (int k = 0; k < n; ++k)
      S.step((R)dt);
  });
}
int pdem_counters(pdem_handle h, pdem_counters_t* out) {
  if (!out) {
    g_err = "counters: null output";
    return PDEM_ERR_INVALID;
  }
  return with(h, [&](auto& S) {
    long sz[3];
    int in[8];
    double mo = 0;
    S.lastCounters(sz, in, &mo);
    out->pairs = sz[0], out->contacts = sz[1], out->manifolds = sz[2];
    out->colors_velocity = in[0], out->colors_position = in[1];
    out->velocity_sweeps = in[2], out->stabilization_sweeps = in[3], out->position_sweeps = in[4];
    out->status = in[5];
    out->color_rounds_velocity = in[6];
    out->color_rounds_position = in[7];
    out->max_overlap = mo;
  });
}
int pdem_step_hertz(pdem_handle h, double dt, int substeps, double skin) {
  BODY(S.stepHertz((R)dt, substeps, (R)skin));
}
int pdem_compute_overlaps(pdem_handle h, double* out) {
  BODY({
    const R v = S.computeOverlaps();
    if (out)
      *out = v;
  });
}
int pdem_num_particles(pdem_handle h) {
  int n = -1;
  with(h, [&](auto& S) { n = S.numParticles(); });
  return n;
}
int pdem_num_contacts(pdem_handle h) {
  int n = -1;
  with(h, [&](auto& S) { n = S.numContacts(); });
  return n;
}
int pdem_num_manifolds(pdem_handle h) {
  int n = -1;
  with(h, [&](auto& S) { n = S.numManifolds(); });
  return n;
}
double pdem_max_overlap(pdem_handle h) {
  double v = 0;
  with(h, [&](auto& S) { v = S.maxOverlap(); });
  return v;
}
int pdem_export_lammps(pdem_handle h, const char* fn, int step) {
  BODY({
    std::vector<double> pos, vel, quat, sc;
    fetch(S, 0, 3, pos);
    fetch(S, 1, 3, vel);
    fetch(S, 2, 4, quat);
    fetch(S, 5, 1, sc);
    std::vector<double> radii(sc.size());
    for (size_t i = 0; i < sc.size(); ++i)
      radii[i] = (double)((R)sc[i] * S.gs_ * S.baseRadius_);
    const bool pbc = S.per_[0] || S.per_[1] || S.per_[2];
    writeLammps(fn, step, pos, vel, quat, radii, pbc);
  });
}
int pdem_write_vtp(pdem_handle h, const char* fn) {
  BODY({
    std::vector<double> pos, vel, sc;
    fetch(S, 0, 3, pos);
    fetch(S, 1, 3, vel);
    fetch(S, 5, 1, sc);
    std::vector<double> radii(sc.size());
    for (size_t i = 0; i < sc.size(); ++i)
      radii[i] = (double)((R)sc[i] * S.gs_ * S.baseRadius_);
    writeVtp(fn, pos, vel, radii);
  });
}

int pdem_get_domain(pdem_handle h, double* mn, double* mx) {
  BODY({
    for (int a = 0; a < 3; ++a)
      mn[a] = (double)S.dmin_[a], mx[a] = (double)S.dmax_[a];
  });
}
int pdem_device_view(pdem_handle h, int field, void** ptr, long* rows, int* row_stride, int* elem_bytes) {
  BODY({
    S.deviceView(field, ptr, rows, row_stride);
    *elem_bytes = (int)sizeof(R);
  });
}
int pdem_scene_block(pdem_handle h, int* block, double* ms, int cap) {
  BODY({
    *block = S.tunedSceneBlock();
    for (int c = 0; c < cap && c < S.kTuneCands; ++c)
      ms[c] = (double)S.tuneMs()[c];
  });
}
int pdem_color_block(pdem_handle h, int* block, double* ms, int cap) {
  BODY({
    *block = S.tunedColorBlock();
    for (int c = 0; c < cap && c < S.kColorTuneCands; ++c)
      ms[c] = (double)S.colorTuneMs()[c];
  });
}
long pdem_get_sdf_grid(pdem_handle h, int rx, int ry, int rz, double* out, long cap) {
  long n = -1;
  const int st = with(h, [&](auto& S) {
    const auto g = S.sdfGrid(rx, ry, rz);
    n = (long)g.size();
    for (long i = 0; i < n && i < cap; ++i)
      out[i] = (double)g[i];
  });
  return st == PDEM_OK ? n : -1;
}
int pdem_export_sdf(pdem_handle h, const char* fn, int rx, int ry, int rz) {
  BODY({
    const auto g = S.sdfGrid(rx, ry, rz);
    const float mn[3] = {(float)S.dmin_[0], (float)S.dmin_[1], (float)S.dmin_[2]};
    const float mx[3] = {(float)S.dmax_[0], (float)S.dmax_[1], (float)S.dmax_[2]};
    writeSdfVti(fn, g, rx, ry, rz, mn, mx);
  });
}

// ---- diagnostics ----
int pdem_debug_counts(pdem_handle h, long* out) { BODY(S.counts(out)); }
long pdem_debug_pairs(pdem_handle h, int* out, long cap) {
  long n = -1;
  with(h, [&](auto& S) { n = S.getPairs(out, cap); });
  return n;
}
long pdem_debug_contacts(pdem_handle h, double* out, long cap) {
  long n = -1;
  with(h, [&](auto& S) { n = S.getContacts(out, cap, false); });
  return n;
}
long pdem_debug_contact_mu(pdem_handle h, double* out, long cap) {
  long n = -1;
  with(h, [&](auto& S) { n = S.getContacts(out, cap, true); });
  return n;
}
long pdem_debug_manifolds(pdem_handle h, double* out, long cap) {
  long n = -1;
  with(h, [&](auto& S) { n = S.getManifolds(out, cap); });
  return n;
}
long pdem_debug_manifold_colors(pdem_handle h, int* out, long cap) {
  long n = -1;
  with(h, [&](auto& S) { n = S.getColors(true, out, cap); });
  return n;
}
long pdem_debug_contact_colors(pdem_handle h, int* out, long cap) {
  long n = -1;
  with(h, [&](auto& S) { n = S.getColors(false, out, cap); });
  return n;
}
long pdem_debug_lambda(pdem_handle h, double* out, long cap) {
  long n = -1;
  with(h, [&](auto& S) { n = S.getLambda(out, cap); });
  return n;
}
long pdem_debug_pair_keys(pdem_handle h, unsigned long long* out, long cap) {
  long n = -1;
  with(h, [&](auto& S) { n = S.getPairKeys(out, cap); });
  return n;
}
long pdem_debug_ledger(pdem_handle h, unsigned long long* keys, double* vals, long cap) {
  long n = -1;
  with(h, [&](auto& S) { n = S.getLedger(keys, vals, cap); });
  return n;
}
long pdem_debug_grounded(pdem_handle h, int* out, long cap) {
  long n = -1;
  with(h, [&](auto& S) { n = S.getGrounded(out, cap); });
  return n;
}
long pdem_debug_pos_lambda(pdem_handle h, double* out, long cap) {
  long n = -1;
  with(h, [&](auto& S) { n = S.getPosLambda(out, cap); });
  return n;
}
long pdem_debug_hertz(pdem_handle h, unsigned long long* keys, double* xi, long cap) {
  long n = -1;
  with(h, [&](auto& S) { n = S.getHertz(keys, xi, cap); });
  return n;
}
int pdem_debug_set_max_contacts(pdem_handle h, int n) { BODY(S.setMaxContacts(n)); }
int pdem_debug_set_barrier_spins(pdem_handle h, long spins) { BODY(S.setBarrierSpins(spins)); }

// ---- batched form ----
int pdem_set_scenes(pdem_handle h, int nscenes, const int* first_body) {
  if (!first_body) {
    g_err = "set_scenes: null scene table";
    return PDEM_ERR_INVALID;
  }
  BODY(S.setScenes(nscenes, first_body));
}
int pdem_set_scene_material(pdem_handle h, int scene, double e_n, double mu) {
  BODY(S.setSceneMaterial(scene, (R)e_n, (R)mu));
}
int pdem_set_wall_scene(pdem_handle h, int wall, int scene) { BODY(S.setWallScene(wall, scene)); }
long pdem_scene_counters(pdem_handle h, double* out, long cap) {
  long n = -1;
  if (with(h, [&](auto& S) { n = S.sceneCounters(out, cap); }) != PDEM_OK)
    return -1;
  return n;
}

// ---- instrumentation ----
int pdem_timer_start(pdem_handle h) { BODY(S.timerStart()); }
int pdem_debug_ranked(pdem_handle h, long* out2) { BODY(out2[0] = S.rankStats_[0]; out2[1] = S.rankStats_[1]); }
int pdem_debug_reuse(pdem_handle h, long* out3) { BODY(for (int i = 0; i < 3; ++i) out3[i] = S.reuse_[i]); }
int pdem_timer_stop(pdem_handle h, double* ms) { BODY(*ms = S.timerStop()); }
long pdem_debug_allocs(void) { return pdem::gDeviceAllocs; }
int pdem_debug_sweeps(pdem_handle h, long* out4) {
  BODY(for (int i = 0; i < 4; ++i) out4[i] = S.sweeps_[i]);
}
int pdem_profile_enable(pdem_handle h, int on) { BODY(S.profileEnable(on != 0)); }
int pdem_profile_read_host(pdem_handle h, double* ms, int cap) {
  int n = -1;
  with(h, [&](auto& S) {
    using T = std::remove_reference_t<decltype(S)>;
    n = T::ST_COUNT;
    for (int i = 0; i < n && i < cap; ++i)
      ms[i] = S.stageHostMs_[i];
  });
  return n;
}
int pdem_profile_read(pdem_handle h, double* ms, long* calls, int cap, long* launches) {
  int n = -1;
  with(h, [&](auto& S) {
    using T = std::remove_reference_t<decltype(S)>;
    n = T::ST_COUNT;
    for (int i = 0; i < n && i < cap; ++i) {
      if (ms)
        ms[i] = S.stageMs_[i];
      if (calls)
        calls[i] = S.stageCalls_[i];
    }
    if (launches)
      *launches = S.launches_;
  });
  return n;
}

int pdem_debug_radix_sort(const unsigned long long* keys, const int* vals, int n, int end_bit,
                          unsigned long long* out_keys, int* out_vals) {
  if (n < 0 || end_bit < 0 || end_bit > 64 || (n > 0 && (!keys || !vals || !out_keys || !out_vals))) {
    g_err = "debug_radix_sort: n >= 0, 0 <= end_bit <= 64 and four arrays";
    return PDEM_ERR_INVALID;
  }
  if (n == 0)
    return PDEM_OK;
  unsigned long long *dk = nullptr, *dko = nullptr, *dkt = nullptr;
  int *dv = nullptr, *dvo = nullptr, *dvt = nullptr, *dh = nullptr;
  cudaError_t e = cudaSuccess;
  const size_t kb = (size_t)n * sizeof(unsigned long long), vb = (size_t)n * sizeof(int);
  for (auto* p : {&dk, &dko, &dkt})
    if (e == cudaSuccess)
      e = cudaMalloc(reinterpret_cast<void**>(p), kb);
  for (auto* p : {&dv, &dvo, &dvt})
    if (e == cudaSuccess)
      e = cudaMalloc(reinterpret_cast<void**>(p), vb);
  if (e == cudaSuccess)
    e = cudaMalloc(reinterpret_cast<void**>(&dh), 256 * (size_t)pdem::radixBlocks(n) * sizeof(int));
  if (e == cudaSuccess)
    e = cudaMemcpy(dk, keys, kb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(dv, vals, vb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = pdem::radixSortPairs(dk, dko, dv, dvo, n, end_bit, dkt, dvt, dh, 0);
  if (e == cudaSuccess)
    e = cudaDeviceSynchronize();
  if (e == cudaSuccess)
    e = cudaMemcpy(out_keys, dko, kb, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess)
    e = cudaMemcpy(out_vals, dvo, vb, cudaMemcpyDeviceToHost);
  for (void* p : {(void*)dk, (void*)dko, (void*)dkt, (void*)dv, (void*)dvo, (void*)dvt, (void*)dh})
    if (p)
      cudaFree(p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    g_err = std::string("debug_radix_sort: ") + cudaGetErrorString(e);
    return PDEM_ERR_CUDA;
  }
  return PDEM_OK;
}

int pdem_xa_begin(pdem_handle h, const double* x, const double* q, const double* v, const double* w, int n) {
  BODY(pdem::xadjBegin(S, x, q, v, w, n));
}
int pdem_xa_step(pdem_handle h, double dt, int substeps) { BODY(pdem::xadjStep(S, dt, substeps)); }
int pdem_xa_state(pdem_handle h, double* x, double* q, double* v, double* w) {
  BODY(pdem::xadjState(S, x, q, v, w));
}
int pdem_xa_backward(pdem_handle h, const double* gx, const double* gq, const double* gv, const double* gw,
                     double* dx, double* dq, double* dv, double* dw, double* dtheta) {
  BODY(pdem::xadjBackward(S, gx, gq, gv, gw, dx, dq, dv, dw, dtheta));
}
int pdem_xa_info(pdem_handle h, long* out, double* err) { BODY(pdem::xadjInfo(S, out, err)); }
int pdem_xa_branches(pdem_handle h, unsigned long long* hash) { BODY(*hash = pdem::xadjBranches(S)); }
long pdem_xa_signature(pdem_handle h, long* out, long cap) {
  long n = -1;
  if (with(h, [&](auto& S) { n = pdem::xadjSignature(S, out, cap); }) != PDEM_OK)
    return -1;
  return n;
}

}  // extern "C"
