// Host check of the XPBD adjoint's hand-written reverses (test infrastructure).
//
// The local maps of csrc/pdem_xadj.cuh are host-and-device code. Compiled here for the host, each
// hand-written reverse (pgsRev, warmRev, vn0Rev, posRev) is compared on random inputs with the
// vector-Jacobian product of its map taken through forward-mode dual numbers (Dd, one chunk of
// lanes at a time). The inputs are drawn so that every branch is visited: side flags, the
// restitution cut-off, clamped and free normal impulses, the friction cone on and off, walls and
// body pairs, active and inactive position contacts. Prints one line per map (cases, branches seen,
// largest relative difference) and exits non-zero when a difference exceeds the tolerance.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <set>

#include "pdem_xadj.cuh"

// (the using-directives stay inside this namespace: at file scope they would make the CUDA host
// headers' own sqrt calls ambiguous)
namespace xcheck {
using namespace pdem;
using namespace pdem::xadj;

template <int NI, int NO, class F>
void dualVjp(const double* in, const double* yb, double* xb, F f) {
  using D = Dd<kLanes>;
  for (int c0 = 0; c0 < NI; c0 += kLanes) {
    D x[NI], y[NO];
    for (int i = 0; i < NI; ++i) {
      x[i] = D(in[i]);
      if (i - c0 >= 0 && i - c0 < kLanes)
        x[i].d[i - c0] = 1.0;
    }
    f(x, y);
    for (int l = 0; l < kLanes && c0 + l < NI; ++l) {
      double s = 0.0;
      for (int o = 0; o < NO; ++o)
        s += yb[o] * y[o].d[l];
      xb[c0 + l] += s;
    }
  }
}

struct Gen {
  std::mt19937_64 rng;
  explicit Gen(unsigned long long seed) : rng(seed) {}
  double u(double a, double b) { return std::uniform_real_distribution<double>(a, b)(rng); }
  double n(double s) { return std::normal_distribution<double>(0.0, s)(rng); }
  int i(int a, int b) { return std::uniform_int_distribution<int>(a, b)(rng); }
  void vec(double* p, double s) { p[0] = n(s), p[1] = n(s), p[2] = n(s); }
  void quat(double* q) {
    double s = 0.0;
    for (int k = 0; k < 4; ++k)
      q[k] = n(1.0), s += q[k] * q[k];
    s = std::sqrt(s);
    for (int k = 0; k < 4; ++k)
      q[k] /= s;
  }
};

double relDiff(const double* a, const double* b, int lo, int hi) {
  double m = 0.0, d = 0.0;
  for (int k = lo; k < hi; ++k) {
    m = std::fmax(m, std::fabs(b[k]));
    d = std::fmax(d, std::fabs(a[k] - b[k]));
  }
  return m > 0.0 ? d / m : d;
}

ManC manifold(Gen& g, bool hasB, int np, int sf) {
  ManC m;
  m.invN = 1.0 / np;
  m.hasB = hasB;
  m.wv = V3<double>{0.0, 0.0, 0.0};
  m.imA = g.u(0.5, 2.0);
  m.imB = hasB ? g.u(0.5, 2.0) : 0.0;
  const double a = g.u(1.0, 3.0), b = g.u(1.0, 3.0);
  m.iIA = V3<double>{a, a, a};
  m.iIB = hasB ? V3<double>{b, b, b} : V3<double>{0.0, 0.0, 0.0};
  m.eAvg = -1.0;
  m.muAvg = -1.0;
  m.sf = sf;
  return m;
}

// a manifold's geometry: np contacts with normals near a common direction, lever arms about 1
void geometry(Gen& g, double* in, int o, int np, bool hasB) {
  double dir[3];
  g.vec(dir, 1.0);
  const double l = std::sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
  double N[3] = {0, 0, 0}, TA[3] = {0, 0, 0}, TB[3] = {0, 0, 0}, rA[3] = {0, 0, 0}, rB[3] = {0, 0, 0};
  for (int c = 0; c < np; ++c) {
    double n[3], ra[3], rb[3];
    for (int k = 0; k < 3; ++k)
      n[k] = -dir[k] / l + g.n(0.05);
    for (int k = 0; k < 3; ++k)
      ra[k] = -n[k] + g.n(0.1), rb[k] = hasB ? n[k] + g.n(0.1) : g.n(1.0);
    const double ta[3] = {ra[1] * n[2] - ra[2] * n[1], ra[2] * n[0] - ra[0] * n[2], ra[0] * n[1] - ra[1] * n[0]};
    const double tb[3] = {-(rb[1] * n[2] - rb[2] * n[1]), -(rb[2] * n[0] - rb[0] * n[2]), -(rb[0] * n[1] - rb[1] * n[0])};
    for (int k = 0; k < 3; ++k)
      N[k] += n[k], TA[k] += ta[k], TB[k] += tb[k], rA[k] += ra[k], rB[k] += rb[k];
  }
  for (int k = 0; k < 3; ++k)
    in[o + k] = N[k], in[o + 3 + k] = TA[k], in[o + 6 + k] = TB[k], in[o + 9 + k] = rA[k], in[o + 12 + k] = rB[k];
}

int run(int argc, char** argv) {
  const int cases = argc > 1 ? std::atoi(argv[1]) : 4000;
  const double tol = 1e-9;
  const double vRest = 0.2;
  Gen g(20261203ull);
  int bad = 0;
  // ---- PGS update ----
  {
    double worst = 0.0;
    std::set<unsigned> seen;
    for (int c = 0; c < cases; ++c) {
      const bool hasB = g.i(0, 3) != 0;
      const int np = hasB ? 1 : g.i(1, 2);
      const int sf = hasB ? (g.i(0, 5) < 4 ? 0 : g.i(1, 2)) : 0;
      const ManC m = manifold(g, hasB, np, sf);
      double in[kPgsIn], out[kPgsOut], yb[kPgsOut], xh[kPgsIn] = {}, xd[kPgsIn] = {};
      for (int k = 0; k < 12; k += 3)
        g.vec(in + k, 0.5);
      in[12] = g.i(0, 2) == 0 ? 0.0 : std::fabs(g.n(0.5));
      if (g.i(0, 1))
        g.vec(in + 13, 0.3);
      else
        in[13] = in[14] = in[15] = 0.0;
      geometry(g, in, 16, np, hasB);
      g.quat(in + 31);
      g.quat(in + 35);
      in[39] = g.n(0.5);
      g.vec(in + 40, 0.3);
      in[43] = g.i(0, 2) == 0 ? 0.0 : g.n(0.5);
      in[44] = g.u(0.0, 1.0);
      in[45] = g.i(0, 2) == 0 ? 0.0 : g.u(0.0, 0.5);
      in[46] = g.i(0, 5) == 0 ? 0.0 : g.u(0.05, 1.0);
      for (int k = 0; k < kPgsOut; ++k)
        yb[k] = g.n(1.0);
      if (!hasB)  // a wall has no second body: its velocity slots carry nothing (as in the kernels)
        for (int k = 6; k < 12; ++k)
          yb[k] = 0.0;
      unsigned bits = 0;
      pgsMap<double>(in, out, m, vRest, &bits);
      seen.insert(bits);
      pgsRev(in, yb, xh, m, vRest);
      dualVjp<kPgsIn, kPgsOut>(in, yb, xd, [&](const Dd<kLanes>* x, Dd<kLanes>* y) { pgsMap(x, y, m, vRest); });
      const double rd = relDiff(xh, xd, 0, kPgsIn);
      if (rd > tol && std::getenv("XADJ_VERBOSE")) {
        std::printf("case %d bits %u hasB %d sf %d np %d:", c, bits, (int)hasB, sf, np);
        for (int k = 0; k < kPgsIn; ++k)
          if (std::fabs(xh[k] - xd[k]) > 1e-9 * (std::fabs(xd[k]) + 1e-9))
            std::printf(" [%d] %.6g/%.6g", k, xh[k], xd[k]);
        std::printf("\n");
      }
      worst = std::fmax(worst, rd);
    }
    std::printf("pgs cases %d branch-sets %zu max-rel %.3e\n", cases, seen.size(), worst);
    bad += worst > tol;
  }
  // ---- warm start (the non-velocity inputs) ----
  {
    double worst = 0.0;
    for (int c = 0; c < cases; ++c) {
      const bool hasB = g.i(0, 3) != 0;
      const int np = hasB ? 1 : g.i(1, 2);
      const ManC m = manifold(g, hasB, np, 0);
      double in[kWarmIn] = {}, yb[kWarmOut], xh[kWarmIn] = {}, xd[kWarmIn] = {};
      in[12] = g.i(0, 2) == 0 ? 0.0 : std::fabs(g.n(0.5));
      if (g.i(0, 1))
        g.vec(in + 13, 0.3);
      geometry(g, in, 16, np, hasB);
      g.quat(in + 31);
      g.quat(in + 35);
      for (int k = 0; k < kWarmOut; ++k)
        yb[k] = g.n(1.0);
      if (!hasB)
        for (int k = 6; k < 12; ++k)
          yb[k] = 0.0;
      warmRev(in, yb, xh, m);
      dualVjp<kWarmIn, kWarmOut>(in, yb, xd, [&](const Dd<kLanes>* x, Dd<kLanes>* y) { warmMap(x, y, m); });
      worst = std::fmax(worst, relDiff(xh, xd, 12, kWarmIn));
    }
    std::printf("warm cases %d max-rel %.3e\n", cases, worst);
    bad += worst > tol;
  }
  // ---- approach velocity ----
  {
    double worst = 0.0;
    for (int c = 0; c < cases; ++c) {
      const bool hasB = g.i(0, 3) != 0;
      const int np = hasB ? 1 : g.i(1, 2);
      const ManC m = manifold(g, hasB, np, 0);
      double in[kVn0In] = {}, yb[kVn0Out], xh[kVn0In] = {}, xd[kVn0In] = {};
      for (int k = 0; k < 12; k += 3)
        g.vec(in + k, 0.5);
      geometry(g, in, 12, np, hasB);
      for (int k = 0; k < kVn0Out; ++k)
        yb[k] = g.n(1.0);
      vn0Rev(in, yb, xh, m);
      dualVjp<kVn0In, kVn0Out>(in, yb, xd, [&](const Dd<kLanes>* x, Dd<kLanes>* y) { vn0Map(x, y, m); });
      // a wall's second-body slots are unused: compare the rest
      double w = std::fmax(relDiff(xh, xd, 0, 6), relDiff(xh, xd, 12, kVn0In));
      if (m.hasB)
        w = std::fmax(w, relDiff(xh, xd, 6, 12));
      worst = std::fmax(worst, w);
    }
    std::printf("vn0 cases %d max-rel %.3e\n", cases, worst);
    bad += worst > tol;
  }
  // ---- position update ----
  {
    double worst = 0.0;
    int active = 0;
    for (int c = 0; c < cases; ++c) {
      PosC pc;
      pc.hasB = g.i(0, 3) != 0;
      pc.imA = g.u(0.5, 2.0);
      pc.imB = pc.hasB ? g.u(0.5, 2.0) : 0.0;
      const double a = g.u(1.0, 3.0), b = g.u(1.0, 3.0);
      pc.iIA = V3<double>{a, a, a};
      pc.iIB = pc.hasB ? V3<double>{b, b, b} : V3<double>{0.0, 0.0, 0.0};
      double in[kPosIn], out[kPosOut], yb[kPosOut], xh[kPosIn] = {}, xd[kPosIn] = {};
      // two unit spheres nearly touching along n (overlapping or not), small rotations of the substep
      double n[3];
      g.vec(n, 1.0);
      const double l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
      for (int k = 0; k < 3; ++k)
        n[k] /= l;
      const double gap = g.n(0.05);
      for (int k = 0; k < 3; ++k) {
        in[k] = 2.0 * n[k] + gap * n[k] + g.n(0.01);  // xA
        in[3 + k] = g.n(0.01);                          // xB
        in[22 + k] = n[k];                              // normal (from B to A)
        in[25 + k] = -n[k];                             // rA
        in[28 + k] = pc.hasB ? n[k] : -0.0 + g.n(0.5);  // rB (a body's lever arm, or a plane point)
      }
      g.quat(in + 14);
      g.quat(in + 18);
      for (int k = 0; k < 4; ++k)
        in[6 + k] = in[14 + k] + g.n(0.01), in[10 + k] = in[18 + k] + g.n(0.01);
      for (int k = 0; k < kPosOut; ++k)
        yb[k] = g.n(1.0);
      unsigned bits = 0;
      posMap<double>(in, out, pc, &bits);
      active += bits == 4u;
      posRev(in, yb, xh, pc);
      dualVjp<kPosIn, kPosOut>(in, yb, xd, [&](const Dd<kLanes>* x, Dd<kLanes>* y) { posMap(x, y, pc); });
      // the second body's position and orientation do not enter a wall contact: skip them there
      double w = relDiff(xh, xd, 0, 3);
      w = std::fmax(w, relDiff(xh, xd, 6, 10));
      w = std::fmax(w, relDiff(xh, xd, 14, 18));
      w = std::fmax(w, relDiff(xh, xd, 22, kPosIn));
      if (pc.hasB) {
        w = std::fmax(w, relDiff(xh, xd, 3, 6));
        w = std::fmax(w, relDiff(xh, xd, 10, 14));
        w = std::fmax(w, relDiff(xh, xd, 18, 22));
      }
      worst = std::fmax(worst, w);
    }
    std::printf("pos cases %d active %d max-rel %.3e\n", cases, active, worst);
    bad += worst > tol;
  }
  return bad ? 1 : 0;
}

}  // namespace xcheck

int main(int argc, char** argv) { return xcheck::run(argc, argv); }
