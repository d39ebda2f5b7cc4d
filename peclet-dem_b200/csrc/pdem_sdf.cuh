// Packed-bed SDF over the domain (get_sdf_grid, src/output_sdf.hpp:25-196): every voxel starts at
// 100; each particle writes min(analytic SDF x scale) over its band (bounding radius x scale x 1.2,
// wrapped on periodic axes, clipped on the others) and marks the voxels nearer than that radius
// fixed; then max(res) x 4 Jacobi Eikonal sweeps (spacing = the x voxel size) fill the rest.
// The particle scale alone sizes the shape (the global scale is not applied) and box shapes
// splat nothing, as in the reference. The minimum is order-free (ordered-bits atomics), so the
// field is deterministic.
#pragma once
#include "pdem_common.cuh"

namespace pdem {

template <class R>
struct SdfGridP {
  int rx, ry, rz, px, py, pz;
  R o[3], vox[3];
};

// min into a float / double through its bit pattern: non-negative values order as signed
// integers, negative ones in reverse as unsigned; -0 is stored as +0
__device__ __forceinline__ void atomicMinReal(float* p, float v) {
  if (v == 0.0f)
    v = 0.0f;
  if (v >= 0.0f)
    atomicMin(reinterpret_cast<int*>(p), __float_as_int(v));
  else
    atomicMax(reinterpret_cast<unsigned*>(p), __float_as_uint(v));
}
__device__ __forceinline__ void atomicMinReal(double* p, double v) {
  if (v == 0.0)
    v = 0.0;
  if (v >= 0.0)
    atomicMin(reinterpret_cast<long long*>(p), __double_as_longlong(v));
  else
    atomicMax(reinterpret_cast<unsigned long long*>(p), (unsigned long long)__double_as_longlong(v));
}

template <class R>
__global__ void kSdfInit(R* grid, int* state, long total) {
  GRID_STRIDE(i, total) {
    grid[i] = R(100);
    state[i] = 0;
  }
}

// one warp per particle; its lanes walk the band's voxels
template <class R>
__global__ void kSdfSplat(Dev<R> d, int numReal, SdfGridP<R> G, R* grid, int* state) {
  const int lane = threadIdx.x & 31;
  for (long i = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < numReal;
       i += ((long)gridDim.x * blockDim.x) >> 5) {
    const V3<R> pw = v3(d.pos[i]);
    const Q4<R> q = d.quat[i];
    const R sc = d.scale[i];
    const ShapeDesc<R> shp = d.shapes[d.shapeId[i]];
    R rbound = R(1);
    if (shp.type == SHAPE_HCYL) {
      const R r = shp.par[0], h = shp.par[1];
      rbound = sqrt(r * r + (h * R(0.5)) * (h * R(0.5)));
    } else if (shp.type == SHAPE_SPHERE || shp.type == SHAPE_GRID) {
      rbound = shp.par[0];
    }
    rbound *= sc;
    rbound *= R(1.2);
    int mn[3], mx[3];
    const R p[3] = {pw.x, pw.y, pw.z};
    const int res[3] = {G.rx, G.ry, G.rz}, per[3] = {G.px, G.py, G.pz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      mn[a] = (int)floor((p[a] - rbound - G.o[a]) / G.vox[a]);
      mx[a] = (int)ceil((p[a] + rbound - G.o[a]) / G.vox[a]);
      if (!per[a]) {
        mn[a] = mn[a] < 0 ? 0 : mn[a];
        mx[a] = mx[a] > res[a] - 1 ? res[a] - 1 : mx[a];
      }
    }
    const long nx = mx[0] - mn[0] + 1, ny = mx[1] - mn[1] + 1, nz = mx[2] - mn[2] + 1;
    const long nv = (nx > 0 && ny > 0 && nz > 0) ? nx * ny * nz : 0;
    const R isc = R(1) / sc;
    for (long t = lane; t < nv; t += 32) {
      const int x = mn[0] + (int)(t % nx), y = mn[1] + (int)((t / nx) % ny), z = mn[2] + (int)(t / (nx * ny));
      if ((!G.px && (x < 0 || x >= G.rx)) || (!G.py && (y < 0 || y >= G.ry)) || (!G.pz && (z < 0 || z >= G.rz)))
        continue;
      const V3<R> vp{G.o[0] + (R(x) + R(0.5)) * G.vox[0], G.o[1] + (R(y) + R(0.5)) * G.vox[1],
                     G.o[2] + (R(z) + R(0.5)) * G.vox[2]};
      const V3<R> pl = mul(invrot(q, sub(vp, pw)), isc);
      R distc = R(100);
      if (shp.type == SHAPE_HCYL)
        distc = sdfHollowCyl(pl, shp.par);
      else if (shp.type == SHAPE_SPHERE)
        distc = sdfSphere(pl, shp.par);
      else if (shp.type == SHAPE_GRID)
        distc = sdfShape(pl, shp, d.sdfGrid);
      const R dist = distc * sc;
      const int wx = (x % G.rx + G.rx) % G.rx, wy = (y % G.ry + G.ry) % G.ry, wz = (z % G.rz + G.rz) % G.rz;
      const long vi = (long)wz * G.rx * G.ry + (long)wy * G.rx + wx;
      atomicMinReal(&grid[vi], dist);
      if (dist < rbound)
        state[vi] = 1;
    }
  }
}

// one Jacobi Eikonal sweep (the fast iterative method's local quadratic solve)
template <class R>
__global__ void kSdfEikonal(SdfGridP<R> G, const R* in, R* out, const int* state, R h) {
  const long sy = G.rx, sz = (long)G.rx * G.ry, total = sz * G.rz;
  GRID_STRIDE(idx, total) {
    if (state[idx] == 1) {
      out[idx] = in[idx];
      continue;
    }
    const int z = (int)(idx / sz);
    const long rem = idx % sz;
    const int y = (int)(rem / sy), x = (int)(rem % sy);
    R xm = 100, xp = 100, ym = 100, yp = 100, zm = 100, zp = 100;
    if (x > 0)
      xm = in[idx - 1];
    else if (G.px)
      xm = in[idx - 1 + G.rx];
    if (x < G.rx - 1)
      xp = in[idx + 1];
    else if (G.px)
      xp = in[idx + 1 - G.rx];
    if (y > 0)
      ym = in[idx - sy];
    else if (G.py)
      ym = in[(long)z * sz + (long)(G.ry - 1) * sy + x];
    if (y < G.ry - 1)
      yp = in[idx + sy];
    else if (G.py)
      yp = in[(long)z * sz + x];
    if (z > 0)
      zm = in[idx - sz];
    else if (G.pz)
      zm = in[(long)(G.rz - 1) * sz + (long)y * sy + x];
    if (z < G.rz - 1)
      zp = in[idx + sz];
    else if (G.pz)
      zp = in[(long)y * sy + x];
    R a = fmin(xm, xp), b = fmin(ym, yp), c = fmin(zm, zp), t;
    if (a > b)
      t = a, a = b, b = t;
    if (b > c)
      t = b, b = c, c = t;
    if (a > b)
      t = a, a = b, b = t;
    R u = 100;
    const R u1 = a + h;
    if (u1 <= b) {
      u = u1;
    } else {
      const R d2 = R(2) * h * h - (a - b) * (a - b);
      const R u2 = (d2 < R(0)) ? R(100) : (a + b + sqrt(d2)) * R(0.5);
      if (u2 <= c) {
        u = u2;
      } else {
        const R s = a + b + c, qd = s * s - R(3) * (a * a + b * b + c * c - h * h);
        u = (qd < R(0)) ? R(100) : (s + sqrt(qd)) / R(3);
      }
    }
    out[idx] = u;
  }
}

}  // namespace pdem
