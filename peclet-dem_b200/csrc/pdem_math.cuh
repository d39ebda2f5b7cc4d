// Device math for the B200 substep: 3-vectors, quaternions and the analytic SDFs.
//
// Every expression keeps the reference's evaluation order (src/dem_portable.hpp:17-113) and the
// library is compiled with -fmad=false, so with R = float the arithmetic matches the reference
// operation for operation and with R = double it matches the FP64 oracle. Vectors are stored in
// 4-wide aligned records (`Q4<R>`: 16 B for float, 32 B for double) so one particle field is one
// aligned load; the fourth lane carries a related scalar where one exists.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pdem {

template <class R>
struct alignas(sizeof(R) * 4) Q4 {
  R x, y, z, w;
};
template <class R>
struct V3 {
  R x, y, z;
};

#define PD __host__ __device__ __forceinline__

template <class R>
PD V3<R> v3(Q4<R> a) {
  return {a.x, a.y, a.z};
}
template <class R>
PD Q4<R> q4(V3<R> a, R w = R(0)) {
  return {a.x, a.y, a.z, w};
}
template <class R>
PD V3<R> add(V3<R> a, V3<R> b) {
  return {a.x + b.x, a.y + b.y, a.z + b.z};
}
template <class R>
PD V3<R> sub(V3<R> a, V3<R> b) {
  return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <class R>
PD V3<R> mul(V3<R> a, R s) {
  return {a.x * s, a.y * s, a.z * s};
}
template <class R>
PD V3<R> neg(V3<R> a) {
  return {-a.x, -a.y, -a.z};
}
template <class R>
PD R dot(V3<R> a, V3<R> b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <class R>
PD R vlen(V3<R> v) {
  return sqrt(dot(v, v));
}
template <class R>
PD V3<R> cross(V3<R> a, V3<R> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R>
PD bool nonzero(V3<R> a) {
  return a.x != R(0) || a.y != R(0) || a.z != R(0);
}
// q = (x, y, z, w); rotate v by q: v + w t + qv x t with t = 2 qv x v
template <class R>
PD V3<R> rot(Q4<R> q, V3<R> v) {
  const V3<R> qv{q.x, q.y, q.z};
  const V3<R> t = mul(cross(qv, v), R(2));
  return add(add(v, mul(t, q.w)), cross(qv, t));
}
template <class R>
PD V3<R> invrot(Q4<R> q, V3<R> v) {
  return rot(Q4<R>{-q.x, -q.y, -q.z, q.w}, v);
}
template <class R>
PD Q4<R> qinv(Q4<R> q) {
  return {-q.x, -q.y, -q.z, q.w};
}
template <class R>
PD Q4<R> qmul(Q4<R> a, Q4<R> b) {
  return {a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
          a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
// angular velocity change of an impulse J applied as torque: R (invI_body * (R^T J))
template <class R>
PD V3<R> angResponse(Q4<R> q, V3<R> J, V3<R> iI) {
  const V3<R> Jl = invrot(q, J);
  return rot(q, V3<R>{Jl.x * iI.x, Jl.y * iI.y, Jl.z * iI.z});
}
// tau^T I_world^-1 tau (isotropic shortcut as in the reference)
template <class R>
PD R genInvMass(V3<R> tau, V3<R> iI, Q4<R> q) {
  if (iI.x == iI.y && iI.y == iI.z)
    return dot(tau, tau) * iI.x;
  const V3<R> t = invrot(q, tau);
  return t.x * t.x * iI.x + t.y * t.y * iI.y + t.z * t.z * iI.z;
}
template <class R>
PD R computeW(V3<R> r, V3<R> d, R im, V3<R> iI) {
  const V3<R> rn = cross(r, d);
  return im + rn.x * rn.x * iI.x + rn.y * rn.y * iI.y + rn.z * rn.z * iI.z;
}

enum ShapeKind : int { SHAPE_GRID = 0, SHAPE_SPHERE = 1, SHAPE_HCYL = 2, SHAPE_BOX = 3 };

template <class R>
struct ShapeDesc {
  int type;
  int numPoints;
  int shellOffset;
  int gridOffset;
  R par[4];
  int nx, ny, nz, pad;
  R gridOrigin[3];
  R gridInvSpacing[3];
  R shellR;  // largest shell-point norm (canonical units, rounded up); 0 without a shell
};

template <class R>
struct WallDesc {
  int nx, ny, nz, gridOffset;
  R origin[3], invSpacing[3], linVel[3], angVel[3], center[3];
  R restitution, friction;
  int materialId, pad;
};

template <class R>
struct PlaneDesc {
  R p[3], n[3];
};

template <class R>
PD R sdfSphere(V3<R> p, const R* par) {
  return vlen(p) - par[0];
}
template <class R>
PD R sdfHollowCyl(V3<R> p, const R* par) {
  const R ro = par[0], h = par[1], th = par[2];
  const R r = sqrt(p.x * p.x + p.z * p.z);
  const R rm = ro - th * R(0.5);
  const R dx = fabs(r - rm) - th * R(0.5);
  const R dy = fabs(p.y) - h * R(0.5);
  const R ox = fmax(dx, R(0)), oy = fmax(dy, R(0));
  const R out = sqrt(ox * ox + oy * oy);
  const R in = fmin(fmax(dx, dy), R(0));
  return out + in;
}
template <class R>
PD R sdfBox(V3<R> p, const R* par) {
  const R dx = fabs(p.x) - par[0];
  const R dy = fabs(p.y) - par[1];
  const R dz = fabs(p.z) - par[2];
  const R ox = fmax(dx, R(0)), oy = fmax(dy, R(0)), oz = fmax(dz, R(0));
  const R out = sqrt(ox * ox + oy * oy + oz * oz);
  const R in = fmin(fmax(dx, fmax(dy, dz)), R(0));
  return out + in;
}

// trilinear grid sample with clamp; sign = +1 adds the residual (object SDF), -1 subtracts it
// (container SDF) — src/narrowphase.hpp:104-131 and :141-167
template <class R>
PD R sampleTrilinear(V3<R> p, const R* origin, const R* inv, int nx, int ny, int nz, const R* grid,
                     R sign) {
  const R fx = (p.x - origin[0]) * inv[0];
  const R fy = (p.y - origin[1]) * inv[1];
  const R fz = (p.z - origin[2]) * inv[2];
  const R cx = fmin(fmax(fx, R(0)), R(nx - 1));
  const R cy = fmin(fmax(fy, R(0)), R(ny - 1));
  const R cz = fmin(fmax(fz, R(0)), R(nz - 1));
  const int ix = (int)cx, iy = (int)cy, iz = (int)cz;
  const int ix1 = ix < nx - 1 ? ix + 1 : ix;
  const int iy1 = iy < ny - 1 ? iy + 1 : iy;
  const int iz1 = iz < nz - 1 ? iz + 1 : iz;
  const R tx = cx - ix, ty = cy - iy, tz = cz - iz;
  const long nxny = (long)nx * ny;
  auto at = [&](int x, int y, int z) { return grid[(long)z * nxny + (long)y * nx + x]; };
  const R c00 = at(ix, iy, iz) * (1 - tx) + at(ix1, iy, iz) * tx;
  const R c10 = at(ix, iy1, iz) * (1 - tx) + at(ix1, iy1, iz) * tx;
  const R c01 = at(ix, iy, iz1) * (1 - tx) + at(ix1, iy, iz1) * tx;
  const R c11 = at(ix, iy1, iz1) * (1 - tx) + at(ix1, iy1, iz1) * tx;
  const R c0 = c00 * (1 - ty) + c10 * ty;
  const R c1 = c01 * (1 - ty) + c11 * ty;
  const R val = c0 * (1 - tz) + c1 * tz;
  const R rx = (inv[0] > R(0)) ? (fx - cx) / inv[0] : R(0);
  const R ry = (inv[1] > R(0)) ? (fy - cy) / inv[1] : R(0);
  const R rz = (inv[2] > R(0)) ? (fz - cz) / inv[2] : R(0);
  const R res = sqrt(rx * rx + ry * ry + rz * rz);
  return sign > R(0) ? val + res : val - res;
}

template <class R>
PD R sdfShape(V3<R> p, const ShapeDesc<R>& d, const R* grid) {
  if (d.type == SHAPE_GRID)
    return sampleTrilinear(p, d.gridOrigin, d.gridInvSpacing, d.nx, d.ny, d.nz, grid + d.gridOffset, R(1));
  if (d.type == SHAPE_SPHERE)
    return sdfSphere(p, d.par);
  if (d.type == SHAPE_HCYL)
    return sdfHollowCyl(p, d.par);
  if (d.type == SHAPE_BOX)
    return sdfBox(p, d.par);
  return R(1e9);
}
template <class R>
PD R sampleWall(V3<R> p, const WallDesc<R>& w, const R* grid) {
  return sampleTrilinear(p, w.origin, w.invSpacing, w.nx, w.ny, w.nz, grid + w.gridOffset, R(-1));
}

// central-difference SDF gradient at canonical point pc, normalized (src/narrowphase.hpp:235-243)
template <class R>
PD V3<R> sdfNormal(V3<R> pc, const ShapeDesc<R>& d, const R* grid, R eps) {
  V3<R> n{sdfShape(V3<R>{pc.x + eps, pc.y, pc.z}, d, grid) - sdfShape(V3<R>{pc.x - eps, pc.y, pc.z}, d, grid),
          sdfShape(V3<R>{pc.x, pc.y + eps, pc.z}, d, grid) - sdfShape(V3<R>{pc.x, pc.y - eps, pc.z}, d, grid),
          sdfShape(V3<R>{pc.x, pc.y, pc.z + eps}, d, grid) - sdfShape(V3<R>{pc.x, pc.y, pc.z - eps}, d, grid)};
  const R l = vlen(n);
  return (l > R(1e-9)) ? mul(n, R(1) / l) : V3<R>{0, 1, 0};
}
template <class R>
PD V3<R> wallGradient(V3<R> p, const WallDesc<R>& w, const R* grid, R h) {
  return V3<R>{sampleWall(V3<R>{p.x + h, p.y, p.z}, w, grid) - sampleWall(V3<R>{p.x - h, p.y, p.z}, w, grid),
               sampleWall(V3<R>{p.x, p.y + h, p.z}, w, grid) - sampleWall(V3<R>{p.x, p.y - h, p.z}, w, grid),
               sampleWall(V3<R>{p.x, p.y, p.z + h}, w, grid) - sampleWall(V3<R>{p.x, p.y, p.z - h}, w, grid)};
}

// pseudo-random JP colouring priority (splitmix32 finalizer of the index, index in the low word)
PD long long colorKey(int idx) {
  unsigned z = static_cast<unsigned>(idx) + 0x9e3779b9u;
  z = (z ^ (z >> 16)) * 0x21f0aaadu;
  z = (z ^ (z >> 15)) * 0x735a2d97u;
  z ^= (z >> 15);
  return (static_cast<long long>(z & 0x7fffffffu) << 32) | static_cast<unsigned>(idx);
}

}  // namespace pdem
