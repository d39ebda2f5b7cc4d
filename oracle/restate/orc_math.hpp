// Oracle restatement (test infrastructure): vector/quaternion math and analytic SDFs.
//
// Restates src/dem_portable.hpp:17-113 for a scalar type R (float reproduces the reference's
// arithmetic operation for operation; double is the FP64 oracle). Every expression keeps the
// reference's evaluation order; the build disables FMA contraction (-ffp-contract=off), so at
// R = float the results are bit-identical to the reference compiled the same way.
#pragma once
#include <cmath>
#include <cstdint>

namespace orc {

template <class R>
struct V3 {
  R x, y, z;
};
template <class R>
struct V4 {
  R x, y, z, w;
};

template <class R>
inline V3<R> add(V3<R> a, V3<R> b) {
  return {a.x + b.x, a.y + b.y, a.z + b.z};
}
template <class R>
inline V3<R> sub(V3<R> a, V3<R> b) {
  return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <class R>
inline V3<R> mul(V3<R> a, R s) {
  return {a.x * s, a.y * s, a.z * s};
}
template <class R>
inline R dot(V3<R> a, V3<R> b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <class R>
inline R len(V3<R> v) {
  return std::sqrt(dot(v, v));
}
template <class R>
inline V3<R> cross(V3<R> a, V3<R> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R>
inline V3<R> neg(V3<R> a) {
  return {-a.x, -a.y, -a.z};
}
// dem_portable.hpp:59-63 — v + w*t + qv x t, t = 2 (qv x v)
template <class R>
inline V3<R> rot(V4<R> q, V3<R> v) {
  const V3<R> qv{q.x, q.y, q.z};
  const V3<R> t = mul(cross(qv, v), R(2));
  return add(add(v, mul(t, q.w)), cross(qv, t));
}
// dem_portable.hpp:64-66
template <class R>
inline V3<R> invrot(V4<R> q, V3<R> v) {
  return rot(V4<R>{-q.x, -q.y, -q.z, q.w}, v);
}
template <class R>
inline V4<R> qinv(V4<R> q) {
  return {-q.x, -q.y, -q.z, q.w};
}
// dem_portable.hpp:70-74
template <class R>
inline V4<R> qmul(V4<R> a, V4<R> b) {
  return {a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
          a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}

enum Kind { GRID = 0, SPHERE = 1, HCYL = 2, BOXK = 3 };

// dem_portable.hpp:79-81
template <class R>
inline R sdfSphere(V3<R> p, V4<R> par) {
  return len(p) - par.x;
}
// dem_portable.hpp:83-93 (cylinder axis = body y)
template <class R>
inline R sdfHollowCyl(V3<R> p, V4<R> par) {
  const R ro = par.x, h = par.y, th = par.z;
  const R r = std::sqrt(p.x * p.x + p.z * p.z);
  const R rm = ro - th * R(0.5);
  const R dx = std::fabs(r - rm) - th * R(0.5);
  const R dy = std::fabs(p.y) - h * R(0.5);
  const R ox = std::fmax(dx, R(0)), oy = std::fmax(dy, R(0));
  const R out = std::sqrt(ox * ox + oy * oy);
  const R in = std::fmin(std::fmax(dx, dy), R(0));
  return out + in;
}
// dem_portable.hpp:95-103
template <class R>
inline R sdfBox(V3<R> p, V4<R> par) {
  const R dx = std::fabs(p.x) - par.x;
  const R dy = std::fabs(p.y) - par.y;
  const R dz = std::fabs(p.z) - par.z;
  const R ox = std::fmax(dx, R(0)), oy = std::fmax(dy, R(0)), oz = std::fmax(dz, R(0));
  const R out = std::sqrt(ox * ox + oy * oy + oz * oz);
  const R in = std::fmin(std::fmax(dx, std::fmax(dy, dz)), R(0));
  return out + in;
}

// narrowphase.hpp:29-39 shape descriptor (analytic fields + grid-SDF fields)
template <class R>
struct Shape {
  int type = SPHERE;
  V4<R> par{1, 0, 0, 0};
  int shellOffset = 0;
  int numPoints = 0;
  int gridOffset = 0;
  int nx = 0, ny = 0, nz = 0;
  V3<R> gridOrigin{0, 0, 0};
  V3<R> gridInvSpacing{0, 0, 0};
};

// narrowphase.hpp:104-131 — trilinear grid SDF, clamp + ADD the residual distance (object SDF)
template <class R>
inline R sampleGrid(V3<R> p, const Shape<R>& d, const R* grid) {
  const R fx = (p.x - d.gridOrigin.x) * d.gridInvSpacing.x;
  const R fy = (p.y - d.gridOrigin.y) * d.gridInvSpacing.y;
  const R fz = (p.z - d.gridOrigin.z) * d.gridInvSpacing.z;
  const R cx = std::fmin(std::fmax(fx, R(0)), R(d.nx - 1));
  const R cy = std::fmin(std::fmax(fy, R(0)), R(d.ny - 1));
  const R cz = std::fmin(std::fmax(fz, R(0)), R(d.nz - 1));
  const int ix = (int)cx, iy = (int)cy, iz = (int)cz;
  const int ix1 = ix < d.nx - 1 ? ix + 1 : ix;
  const int iy1 = iy < d.ny - 1 ? iy + 1 : iy;
  const int iz1 = iz < d.nz - 1 ? iz + 1 : iz;
  const R tx = cx - ix, ty = cy - iy, tz = cz - iz;
  const long nxny = (long)d.nx * d.ny;
  auto at = [&](int x, int y, int z) { return grid[d.gridOffset + (long)z * nxny + (long)y * d.nx + x]; };
  const R c00 = at(ix, iy, iz) * (1 - tx) + at(ix1, iy, iz) * tx;
  const R c10 = at(ix, iy1, iz) * (1 - tx) + at(ix1, iy1, iz) * tx;
  const R c01 = at(ix, iy, iz1) * (1 - tx) + at(ix1, iy, iz1) * tx;
  const R c11 = at(ix, iy1, iz1) * (1 - tx) + at(ix1, iy1, iz1) * tx;
  const R c0 = c00 * (1 - ty) + c10 * ty;
  const R c1 = c01 * (1 - ty) + c11 * ty;
  const R val = c0 * (1 - tz) + c1 * tz;
  const R rx = (d.gridInvSpacing.x > R(0)) ? (fx - cx) / d.gridInvSpacing.x : R(0);
  const R ry = (d.gridInvSpacing.y > R(0)) ? (fy - cy) / d.gridInvSpacing.y : R(0);
  const R rz = (d.gridInvSpacing.z > R(0)) ? (fz - cz) / d.gridInvSpacing.z : R(0);
  return val + std::sqrt(rx * rx + ry * ry + rz * rz);
}

// narrowphase.hpp:59-76 static world-space SDF wall
template <class R>
struct Wall {
  int nx = 0, ny = 0, nz = 0;
  int gridOffset = 0;
  V3<R> origin{0, 0, 0};
  V3<R> invSpacing{0, 0, 0};
  V3<R> linVel{0, 0, 0};
  V3<R> angVel{0, 0, 0};
  V3<R> center{0, 0, 0};
  R restitution = 0;
  R friction = 0;
  int materialId = -1;
};

// narrowphase.hpp:141-167 — same trilinear sample, SUBTRACT the residual (container SDF)
template <class R>
inline R sampleWall(V3<R> p, const Wall<R>& w, const R* grid) {
  const R fx = (p.x - w.origin.x) * w.invSpacing.x;
  const R fy = (p.y - w.origin.y) * w.invSpacing.y;
  const R fz = (p.z - w.origin.z) * w.invSpacing.z;
  const R cx = std::fmin(std::fmax(fx, R(0)), R(w.nx - 1));
  const R cy = std::fmin(std::fmax(fy, R(0)), R(w.ny - 1));
  const R cz = std::fmin(std::fmax(fz, R(0)), R(w.nz - 1));
  const int ix = (int)cx, iy = (int)cy, iz = (int)cz;
  const int ix1 = ix < w.nx - 1 ? ix + 1 : ix;
  const int iy1 = iy < w.ny - 1 ? iy + 1 : iy;
  const int iz1 = iz < w.nz - 1 ? iz + 1 : iz;
  const R tx = cx - ix, ty = cy - iy, tz = cz - iz;
  const long nxny = (long)w.nx * w.ny;
  auto at = [&](int x, int y, int z) { return grid[w.gridOffset + (long)z * nxny + (long)y * w.nx + x]; };
  const R c00 = at(ix, iy, iz) * (1 - tx) + at(ix1, iy, iz) * tx;
  const R c10 = at(ix, iy1, iz) * (1 - tx) + at(ix1, iy1, iz) * tx;
  const R c01 = at(ix, iy, iz1) * (1 - tx) + at(ix1, iy, iz1) * tx;
  const R c11 = at(ix, iy1, iz1) * (1 - tx) + at(ix1, iy1, iz1) * tx;
  const R c0 = c00 * (1 - ty) + c10 * ty;
  const R c1 = c01 * (1 - ty) + c11 * ty;
  const R val = c0 * (1 - tz) + c1 * tz;
  const R rx = (w.invSpacing.x > R(0)) ? (fx - cx) / w.invSpacing.x : R(0);
  const R ry = (w.invSpacing.y > R(0)) ? (fy - cy) / w.invSpacing.y : R(0);
  const R rz = (w.invSpacing.z > R(0)) ? (fz - cz) / w.invSpacing.z : R(0);
  return val - std::sqrt(rx * rx + ry * ry + rz * rz);
}

// narrowphase.hpp:171-175 + dem_portable.hpp:105-113
template <class R>
inline R sdfShape(V3<R> p, const Shape<R>& d, const R* grid) {
  if (d.type == GRID)
    return sampleGrid(p, d, grid);
  if (d.type == SPHERE)
    return sdfSphere(p, d.par);
  if (d.type == HCYL)
    return sdfHollowCyl(p, d.par);
  if (d.type == BOXK)
    return sdfBox(p, d.par);
  return R(1e9);
}

}  // namespace orc
