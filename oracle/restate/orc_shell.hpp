// Oracle restatement (test infrastructure): surface point shells of the analytic shapes.
//
// Restates src/shapes_portable.hpp:21-111 (genCylinderShell / genBoxShell). The shell points are part
// of the shape's definition, so they are generated in single precision with the reference's exact
// mixed float/double expression types (M_PI promotes to double, std::cos/sin of a float are the
// float overloads) and are then widened to the working precision.
#pragma once
#include <cmath>
#include <vector>

namespace orc {

struct P3f {
  float x, y, z;
};

// shapes_portable.hpp:21-76: outer wall, inner wall (if thick), annular caps top/bottom
inline std::vector<P3f> cylinderShell(float radius, float height, float thickness, float spacing) {
  std::vector<P3f> out;
  const float ro = radius, ri = radius - thickness, h = height;
  auto ring = [&](float r, int nAng, int nVert) {
    for (int i = 0; i < nAng; ++i) {
      const float th = 2.0f * M_PI * i / nAng;
      for (int j = 0; j <= nVert; ++j) {
        const float y = -0.5f * h + h * j / nVert;
        out.push_back({r * std::cos(th), y, r * std::sin(th)});
      }
    }
  };
  float circ = 2.0f * M_PI * ro;
  int nAng = std::ceil(circ / spacing);
  const int nVert = std::ceil(h / spacing);
  ring(ro, nAng, nVert);
  if (thickness > 0.0f) {
    circ = 2.0f * M_PI * ri;
    nAng = std::ceil(circ / spacing);
    ring(ri, nAng, nVert);
  }
  const float dr = spacing;
  const int nRad = std::ceil(thickness / dr);
  for (int i = 0; i <= nRad; ++i) {
    const float r = ri + (ro - ri) * i / nRad;
    circ = 2.0f * M_PI * r;
    nAng = std::ceil(circ / spacing);
    for (int j = 0; j < nAng; ++j) {
      const float th = 2.0f * M_PI * j / nAng;
      const float x = r * std::cos(th), z = r * std::sin(th);
      out.push_back({x, 0.5f * h, z});
      out.push_back({x, -0.5f * h, z});
    }
  }
  return out;
}

// shapes_portable.hpp:80-111: six face grids whose end points land on the edges
inline std::vector<P3f> boxShell(float hx, float hy, float hz, float spacing) {
  std::vector<P3f> out;
  auto segs = [&](float half) {
    const int n = (int)std::ceil(2.0f * half / spacing);
    return n < 1 ? 1 : n;
  };
  const int nx = segs(hx), ny = segs(hy), nz = segs(hz);
  auto at = [](float half, int i, int n) { return -half + 2.0f * half * (float)i / (float)n; };
  for (int j = 0; j <= ny; ++j)
    for (int k = 0; k <= nz; ++k) {
      const float y = at(hy, j, ny), z = at(hz, k, nz);
      out.push_back({hx, y, z});
      out.push_back({-hx, y, z});
    }
  for (int i = 0; i <= nx; ++i)
    for (int k = 0; k <= nz; ++k) {
      const float x = at(hx, i, nx), z = at(hz, k, nz);
      out.push_back({x, hy, z});
      out.push_back({x, -hy, z});
    }
  for (int i = 0; i <= nx; ++i)
    for (int j = 0; j <= ny; ++j) {
      const float x = at(hx, i, nx), y = at(hy, j, ny);
      out.push_back({x, y, hz});
      out.push_back({x, y, -hz});
    }
  return out;
}

}  // namespace orc
