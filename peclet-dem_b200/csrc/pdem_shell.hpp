// Surface point shells of the analytic shapes (src/shapes_portable.hpp:21-111).
//
// The shell is part of the shape definition, so it is generated exactly as the reference does it:
// single precision, with the reference's mixed float/double expression types (2*pi*r evaluated in
// double then rounded; std::cos/std::sin of a float are the float overloads), then widened. Any
// other rounding would move the probe points and change which contacts exist.
#pragma once
#include <cmath>
#include <vector>

namespace pdem {

struct ShellPoint {
  float x, y, z;
};

// hollow cylinder, axis = body y: outer wall, inner wall (if thick), annular caps at y = +-h/2
inline std::vector<ShellPoint> hollowCylinderShell(float radius, float height, float thickness, float spacing) {
  std::vector<ShellPoint> pts;
  const float rOut = radius, rIn = radius - thickness;
  const int rows = std::ceil(height / spacing);  // axial segments
  auto wall = [&](float r) {
    const float circumference = 2.0f * M_PI * r;
    const int sectors = std::ceil(circumference / spacing);
    for (int a = 0; a < sectors; ++a) {
      const float theta = 2.0f * M_PI * a / sectors;
      for (int b = 0; b <= rows; ++b) {
        const float y = -0.5f * height + height * b / rows;
        pts.push_back({r * std::cos(theta), y, r * std::sin(theta)});
      }
    }
  };
  wall(rOut);
  if (thickness > 0.0f)
    wall(rIn);
  const int rings = std::ceil(thickness / spacing);
  for (int a = 0; a <= rings; ++a) {
    const float r = rIn + (rOut - rIn) * a / rings;
    const float circumference = 2.0f * M_PI * r;
    const int sectors = std::ceil(circumference / spacing);
    for (int b = 0; b < sectors; ++b) {
      const float theta = 2.0f * M_PI * b / sectors;
      const float x = r * std::cos(theta), z = r * std::sin(theta);
      pts.push_back({x, 0.5f * height, z});
      pts.push_back({x, -0.5f * height, z});
    }
  }
  return pts;
}

// axis-aligned box: six face grids with end points on the edges (corners included)
inline std::vector<ShellPoint> boxShell(float hx, float hy, float hz, float spacing) {
  std::vector<ShellPoint> pts;
  auto segments = [&](float half) {
    const int n = (int)std::ceil(2.0f * half / spacing);
    return n < 1 ? 1 : n;
  };
  const int sx = segments(hx), sy = segments(hy), sz = segments(hz);
  auto coord = [](float half, int i, int n) { return -half + 2.0f * half * (float)i / (float)n; };
  for (int j = 0; j <= sy; ++j)
    for (int k = 0; k <= sz; ++k) {
      const float y = coord(hy, j, sy), z = coord(hz, k, sz);
      pts.push_back({hx, y, z});
      pts.push_back({-hx, y, z});
    }
  for (int i = 0; i <= sx; ++i)
    for (int k = 0; k <= sz; ++k) {
      const float x = coord(hx, i, sx), z = coord(hz, k, sz);
      pts.push_back({x, hy, z});
      pts.push_back({x, -hy, z});
    }
  for (int i = 0; i <= sx; ++i)
    for (int j = 0; j <= sy; ++j) {
      const float x = coord(hx, i, sx), y = coord(hy, j, sy);
      pts.push_back({x, y, hz});
      pts.push_back({x, y, -hz});
    }
  return pts;
}

}  // namespace pdem
