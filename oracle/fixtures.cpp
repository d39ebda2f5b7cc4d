// TEST INFRASTRUCTURE ONLY: regenerates the inputs of two of the reference's own unit-test fixtures
// with their seeds and distributions, runs the reference's UNMODIFIED kernels on them (its headers
// compiled against the Kokkos shim, serial flavour), and writes inputs and outputs as raw arrays
// for tests/golden/make_fixtures.py.
//
//   bp_*  tests/arborx/test_broadphase_arborx.cpp:23-101: 4,000 bodies, the last 400 ghosts (hit
//         but issue no query), std::mt19937(12345), positions U[0, 20)^3 and radii U[0.3, 0.7]
//         drawn x, y, z, r per body, margin 0.05. Output: the pair set of its brute-force check
//         (i real, i < j, |x_i - x_j| <= (r_i + margin) + (r_j + margin) per axis, in float),
//         which the reference's broadphase must equal, and the pairs findCollisionsArborX returns.
//   np_*  tests/kokkos/test_narrowphase.cpp:56-96: a 6 x 6 x 6 jittered grid of spheres (global
//         scale 0.7, spacing 1.8 x 0.7, lifted by 0.7 onto a z = 0 plane), std::mt19937(7),
//         jitter U(-0.02, 0.02) per axis, orientations from four N(0, 1) draws normalised, two
//         sphere shapes (radius 1.0 for even ids, 1.02 for odd), margin 0.1 x 0.7, all i < j
//         pairs. Output: the contacts of detectContactsKokkos then detectBoundaryKokkos.
//
//   ref_fixtures <out_dir>
#include <cmath>
#include <cstdio>
#include <random>
#include <string>
#include <vector>

#include <Kokkos_Core.hpp>
#include "broadphase_arborx.hpp"
#include "narrowphase.hpp"

using namespace peclet::dem;

template <class T>
static void put(const std::string& dir, const char* name, const std::vector<T>& v) {
  const std::string path = dir + "/" + name;
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) {
    std::perror(path.c_str());
    std::exit(1);
  }
  if (!v.empty())
    std::fwrite(v.data(), sizeof(T), v.size(), f);
  std::fclose(f);
}

static void broadphaseFixture(const std::string& dir) {
  const int n = 4000, nReal = 3600;
  const float margin = 0.05f, boxL = 20.0f;
  std::vector<float> x(n), y(n), z(n), r(n);
  std::mt19937 rng(12345);
  std::uniform_real_distribution<float> upos(0.f, boxL);
  std::uniform_real_distribution<float> urad(0.3f, 0.7f);
  for (int i = 0; i < n; ++i) {
    x[i] = upos(rng);
    y[i] = upos(rng);
    z[i] = upos(rng);
    r[i] = urad(rng);
  }
  Kokkos::View<float* [3], BpMem> pos("pos", n);
  Kokkos::View<float*, BpMem> rad("rad", n);
  for (int i = 0; i < n; ++i) {
    pos(i, 0) = x[i];
    pos(i, 1) = y[i];
    pos(i, 2) = z[i];
    rad(i) = r[i];
  }
  const int cap = n * 64;
  Kokkos::View<int* [2], BpMem> out("pairs", cap);
  Kokkos::View<int, BpMem> count("count");
  const int got = findCollisionsArborX(pos, rad, n, nReal, margin, out, count);
  std::vector<int> gotPairs;
  for (int k = 0; k < got && k < cap; ++k) {
    gotPairs.push_back(out(k, 0));
    gotPairs.push_back(out(k, 1));
  }
  std::vector<int> brute;
  for (int i = 0; i < nReal; ++i) {
    const float bi = r[i] + margin;
    for (int j = i + 1; j < n; ++j) {
      const float s = bi + (r[j] + margin);
      if (std::fabs(x[i] - x[j]) <= s && std::fabs(y[i] - y[j]) <= s && std::fabs(z[i] - z[j]) <= s) {
        brute.push_back(i);
        brute.push_back(j);
      }
    }
  }
  std::vector<float> xyzr;
  for (int i = 0; i < n; ++i)
    xyzr.insert(xyzr.end(), {x[i], y[i], z[i], r[i]});
  put(dir, "bp_xyzr.f32", xyzr);
  put(dir, "bp_meta.f32", std::vector<float>{(float)n, (float)nReal, margin});
  put(dir, "bp_brute.i32", brute);
  put(dir, "bp_pairs.i32", gotPairs);
  std::printf("broadphase fixture: %d bodies (%d real), %zu brute-force pairs, %zu returned\n", n, nReal,
              brute.size() / 2, gotPairs.size() / 2);
}

static void narrowphaseFixture(const std::string& dir) {
  const int G = 6, N = G * G * G;
  const float gs = 0.7f, spacing = 1.8f * gs, margin = 0.1f * gs;
  std::mt19937 rng(7);
  std::uniform_real_distribution<float> jit(-0.02f, 0.02f);
  std::normal_distribution<float> nq(0.f, 1.f);
  Kokkos::View<float* [3], CpMem> pos("pos", N);
  Kokkos::View<float* [4], CpMem> quat("quat", N);
  Kokkos::View<float*, CpMem> scale("scale", N);
  Kokkos::View<int*, CpMem> sid("sid", N);
  std::vector<float> state;  // x y z qx qy qz qw shape-id per body
  for (int i = 0; i < N; ++i) {
    const int ix = i % G, iy = (i / G) % G, iz = i / (G * G);
    pos(i, 0) = ix * spacing + jit(rng);
    pos(i, 1) = iy * spacing + jit(rng);
    pos(i, 2) = iz * spacing + gs + jit(rng);
    const float a = nq(rng), b = nq(rng), c = nq(rng), d = nq(rng);
    const float nrm = std::sqrt(a * a + b * b + c * c + d * d) + 1e-12f;
    quat(i, 0) = a / nrm;
    quat(i, 1) = b / nrm;
    quat(i, 2) = c / nrm;
    quat(i, 3) = d / nrm;
    scale(i) = 1.0f;
    sid(i) = i & 1;
    state.insert(state.end(), {pos(i, 0), pos(i, 1), pos(i, 2), quat(i, 0), quat(i, 1), quat(i, 2), quat(i, 3),
                               (float)sid(i)});
  }
  Kokkos::View<ShapeDesc*, CpMem> shapes("shapes", 2);
  shapes(0) = ShapeDesc{SPHERE, F4{1.00f, 0, 0, 0}, 0, 0};
  shapes(1) = ShapeDesc{SPHERE, F4{1.02f, 0, 0, 0}, 0, 0};
  Kokkos::View<PlaneP*, CpMem> planes("planes", 1);
  planes(0) = PlaneP{F3{0, 0, 0}, F3{0, 0, 1}};
  Kokkos::View<float* [3], CpMem> shell("shell", 1);
  std::vector<int> pa, pb;
  for (int i = 0; i < N; ++i)
    for (int j = i + 1; j < N; ++j) {
      pa.push_back(i);
      pb.push_back(j);
    }
  const int np = (int)pa.size();
  Kokkos::View<int* [2], CpMem> pairs("pairs", np);
  for (int k = 0; k < np; ++k) {
    pairs(k, 0) = pa[k];
    pairs(k, 1) = pb[k];
  }
  const int cap = N * 32;
  Kokkos::View<ContactC*, CpMem> contacts("contacts", cap);
  Kokkos::View<int, CpMem> count("count");
  Kokkos::View<float, CpMem> maxOv("maxov");
  detectContactsKokkos(pairs, np, pos, quat, scale, sid, shapes, shell, gs, margin, contacts, count, maxOv);
  detectBoundaryKokkos(N, 1, pos, quat, scale, sid, shapes, shell, planes, gs, margin, contacts, count, maxOv);
  int nc = 0;
  Kokkos::deep_copy(nc, count);
  std::vector<int> ab;
  std::vector<float> geo;  // n[3] rA[3] rB[3] dist per contact
  for (int k = 0; k < nc && k < cap; ++k) {
    const ContactC& c = contacts(k);
    ab.insert(ab.end(), {c.bodyA, c.bodyB});
    geo.insert(geo.end(), {c.normal.x, c.normal.y, c.normal.z, c.rA.x, c.rA.y, c.rA.z, c.rB.x, c.rB.y, c.rB.z,
                           c.dist});
  }
  put(dir, "np_state.f32", state);
  put(dir, "np_meta.f32", std::vector<float>{(float)N, gs, margin, 1.00f, 1.02f});
  put(dir, "np_ab.i32", ab);
  put(dir, "np_geo.f32", geo);
  std::printf("narrowphase fixture: %d spheres, %d contacts\n", N, nc);
}

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s <out_dir>\n", argv[0]);
    return 2;
  }
  Kokkos::initialize(argc, argv);
  broadphaseFixture(argv[1]);
  narrowphaseFixture(argv[1]);
  Kokkos::finalize();
  return 0;
}
