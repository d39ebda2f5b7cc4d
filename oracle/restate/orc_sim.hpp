// Oracle restatement (test infrastructure, never shipped): the demStep XPBD substep, the
// Hertz-Mindlin engine and the Simulation facade state, restated serially for a scalar type R.
//
// Each function names the reference function and file:line it follows. The serial loops run in
// ascending index order, so every "atomic" accumulation of the reference happens in ascending source
// index — the canonical order the B200 implementation reproduces. At R = float the results are
// bit-identical to the reference headers compiled against the serial Kokkos shim (the tests check
// this); at R = double this is the FP64 oracle of the B200 FP64 step. Stabilization modes
// "multilevel" (2) and "ordered" (4) are restated.
#pragma once
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <limits>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "orc_math.hpp"
#include "orc_shell.hpp"

namespace orc {

constexpr int kMaxMaterials = 8;
constexpr int kHertzMaxWalls = 4;
using u64 = unsigned long long;

template <class R>
struct Contact {  // contact_preprocessing.hpp:31-45
  int a = 0, b = 0;
  V3<R> n{0, 0, 0}, rA{0, 0, 0}, rB{0, 0, 0};
  R dist = 0, lamN = 0, weight = 0;
  V3<R> bvel{0, 0, 0};
  R e = R(-1), mu = R(-1);
};
template <class R>
struct Manifold {  // contact_preprocessing.hpp:48-63
  int a = 0, b = 0;
  V3<R> N{0, 0, 0}, TA{0, 0, 0}, TB{0, 0, 0}, rA{0, 0, 0}, rB{0, 0, 0};
  int np = 0;
  V3<R> wv{0, 0, 0};
  R e = 0, mu = 0;
};

template <class R>
struct Plane {
  V3<R> p, n;
};

template <class R>
class Sim {
 public:
  // ---------------- state (src/particles.hpp:23-192) ----------------
  int capacity = 0, numReal = 0, numParticles = 0, maxPairs = 0, maxContacts = 0;
  std::vector<V3<R>> pos, vel, angVel, invI, posPred, velPred, angVelPred, deltaPos, deltaVel,
      deltaAngVel, extForce;
  std::vector<V4<R>> quat, quatPred;
  std::vector<R> invMass, scale, targetScale, rad;
  std::vector<int> shapeId, constraintCounts, realIdx;
  std::vector<R> planeFric;  // [cap][2]
  std::vector<unsigned char> grounded, materialId;
  std::vector<long long> bodyWinner;
  std::vector<u64> bodyMask;

  std::vector<int> pairs;  // [maxPairs][2]
  std::vector<Contact<R>> contacts;
  std::vector<Manifold<R>> manifolds;
  std::vector<int> mColor, cColor, contactSlot;
  std::vector<u64> pairKeys, prevPairKeys;
  std::vector<unsigned char> persistent, sideFlags;
  std::vector<R> lambdaAcc, prevLambda, vn0, posLambdaContact, posImpulse, prevPosImpulse;
  std::vector<V3<R>> lambdaT, prevLambdaT, vt0;
  int prevPairCount = 0;
  int pairCount = 0, contactCount = 0, manifoldCount = 0, topGhost = 0;
  R maxOverlap = 0, maxApproach = 0;

  std::vector<Shape<R>> shapes{Shape<R>{}};
  std::vector<V3<R>> shell{V3<R>{0, 0, 0}};
  std::vector<R> sdfGrid{R(0)};
  std::vector<Plane<R>> planes;
  int planeCap = 8;
  std::vector<Wall<R>> walls;
  std::vector<R> wallGrid{R(0)};
  std::vector<R> pairMat;  // [K*K*2], empty = off
  R wallFrictionMax = 0;

  // domain + parameters
  V3<R> dmin{0, 0, 0}, dmax{0, 0, 0}, dsize{0, 0, 0};
  bool px = false, py = false, pz = false;
  V3<R> gravity{0, 0, 0};
  R dt = R(1e-3), globalScale = 1, growthRate = 0, growthFactor = -1, baseRadius = 1;
  R thermoTau = 0, thermoTemp = 0, thermoKB = 1;
  R mu = 0, eN = 0, eT = 0, skin = R(0.1);
  int posIters = 10, velIters = 0;
  bool useGS = true;
  int stabMode = 1;
  int shellPoints = 0;
  V3<R> defaultInvI{R(2.5), R(2.5), R(2.5)};

  // Hertz engine (src/particles.hpp:113-130)
  std::vector<V3<R>> hzXi, hzPrevXi, hzXiWall, hzRefPos;
  std::vector<u64> hzKeys, hzPrevKeys;
  std::vector<R> hzSnPair, hzSnWall, hzE, hzNu;
  std::vector<int> hzWallCand;
  int hzNumWallCand = 0, hzNumPairs = -1, hzPrevCount = 0;
  R hzContactRadiusFrac = R(0.5);

  // ---------------- construction (src/sim.hpp:911-916, particles.hpp:194-288) ----------------
  explicit Sim(int cap) {
    allocate(cap, cap * 64, cap * 16);
    initializeShape(SPHERE, 1, 0, 0);
  }

  void allocate(int cap, int mp, int mc) {
    capacity = cap;
    maxPairs = mp;
    maxContacts = mc;
    auto z3 = V3<R>{0, 0, 0};
    for (auto* v : {&pos, &vel, &angVel, &invI, &posPred, &velPred, &angVelPred, &deltaPos,
                    &deltaVel, &deltaAngVel, &extForce})
      v->assign(cap, z3);
    quat.assign(cap, V4<R>{0, 0, 0, 0});
    quatPred.assign(cap, V4<R>{0, 0, 0, 0});
    for (auto* v : {&invMass, &scale, &targetScale, &rad})
      v->assign(cap, R(0));
    shapeId.assign(cap, 0);
    constraintCounts.assign(cap, 0);
    realIdx.assign(cap, 0);
    planeFric.assign(2 * cap, R(0));
    grounded.assign(cap, 0);
    materialId.assign(cap, 0);
    bodyWinner.assign(cap, 0);
    bodyMask.assign(cap, 0);
    pairs.assign(2 * mp, 0);
    allocContactBuffers(mc);
    hzXiWall.assign((size_t)cap * kHertzMaxWalls, z3);
    hzSnWall.assign((size_t)cap * kHertzMaxWalls, R(0));
    hzWallCand.assign((size_t)cap * 2, 0);
    hzRefPos.assign(cap, z3);
    hzE.assign(8, R(1.0e9));
    hzNu.assign(8, R(0.25));
  }
  void allocContactBuffers(int mc) {
    maxContacts = mc;
    contacts.assign(mc, Contact<R>{});
    manifolds.assign(mc, Manifold<R>{});
    for (auto* v : {&mColor, &cColor, &contactSlot})
      v->assign(mc, 0);
    pairKeys.assign(mc, 0);
    prevPairKeys.assign(mc, 0);
    persistent.assign(mc, 0);
    sideFlags.assign(mc, 0);
    for (auto* v : {&lambdaAcc, &prevLambda, &vn0, &posLambdaContact, &posImpulse, &prevPosImpulse})
      v->assign(mc, R(0));
    for (auto* v : {&lambdaT, &prevLambdaT, &vt0})
      v->assign(mc, V3<R>{0, 0, 0});
  }

  // particles.hpp:297-327 (materialId is grown here too: the reference leaves it at the
  // construction size, which only matters for periodic ghosts with a pair-material table)
  void ensureCapacity(int nc) {
    if (nc <= capacity)
      return;
    auto z3 = V3<R>{0, 0, 0};
    for (auto* v : {&pos, &vel, &angVel, &invI, &posPred, &velPred, &angVelPred, &deltaPos,
                    &deltaVel, &deltaAngVel, &extForce})
      v->resize(nc, z3);
    quat.resize(nc, V4<R>{0, 0, 0, 0});
    quatPred.resize(nc, V4<R>{0, 0, 0, 0});
    for (auto* v : {&invMass, &scale, &targetScale, &rad})
      v->resize(nc, R(0));
    shapeId.resize(nc, 0);
    constraintCounts.resize(nc, 0);
    realIdx.resize(nc, 0);
    planeFric.resize(2 * (size_t)nc, R(0));
    grounded.resize(nc, 0);
    materialId.resize(nc, 0);
    bodyWinner.resize(nc, 0);
    bodyMask.resize(nc, 0);
    capacity = nc;
  }

  // sim.hpp:1620-1654
  void ensureContactCapacity() {
    const int perParticle = std::max(16, shellPoints);
    const long want = (long)capacity * perParticle + (long)capacity * std::max(1, shellPoints) * (long)walls.size();
    if (want > maxContacts) {
      allocContactBuffers((int)want);
      prevPairCount = 0;
    }
  }

  // ---------------- facade setters (src/sim.hpp:943-1424) ----------------
  // sim.hpp:949-1021
  void initializeShape(int type, R radius, R height, R thick) {
    baseRadius = radius;
    V4<R> par{radius, 0, 0, 0};
    std::vector<P3f> sh;
    if (type == HCYL) {
      par = V4<R>{radius, height, thick, 0};
      const float rf = (float)radius, tf = (float)thick;
      float minDim = std::min(rf, tf);
      if (minDim < 1e-4f)
        minDim = rf;
      float sp = std::min(rf * 0.3f, minDim * 0.5f);
      if (sp < 1e-3f)
        sp = 1e-3f;
      sh = cylinderShell(rf, (float)height, tf, sp);
    } else if (type == BOXK) {
      par = V4<R>{radius, radius, radius, 0};
      const float sp = std::max((float)radius * 0.5f, 1e-3f);
      sh = boxShell((float)radius, (float)radius, (float)radius, sp);
    } else {
      type = SPHERE;
      par = V4<R>{radius, 0, 0, 0};
    }
    const int n = (int)sh.size();
    shellPoints = n;
    if (n > 0) {
      shell.resize(n);
      for (int i = 0; i < n; ++i)
        shell[i] = V3<R>{R(sh[i].x), R(sh[i].y), R(sh[i].z)};
    }
    Shape<R> d;
    d.type = type;
    d.par = par;
    d.shellOffset = 0;
    d.numPoints = n;
    shapes[0] = d;
    R ix = 1, iy = 1, iz = 1;
    if (type == SPHERE) {
      if (baseRadius > R(0)) {
        const R v = R(2.5) / (baseRadius * baseRadius);
        ix = iy = iz = v;
      }
    } else if (type == HCYL) {
      const R ro = baseRadius;
      R ri = baseRadius - thick;
      if (ri < 0)
        ri = 0;
      const R tr = ro * ro + ri * ri;
      const R Izz = R(0.5) * tr;
      const R Ixx = (R(1.0) / R(12.0)) * (R(3.0) * tr + height * height);
      if (Ixx > R(1e-6)) {
        ix = R(1.0) / Ixx;
        iy = R(1.0) / Ixx;
      }
      if (Izz > R(1e-6))
        iz = R(1.0) / Izz;
    } else if (type == BOXK) {
      const R L = R(2.0) * baseRadius;
      const R I = (R(1.0) / R(6.0)) * L * L;
      if (I > R(1e-6))
        ix = iy = iz = R(1.0) / I;
    }
    defaultInvI = V3<R>{ix, iy, iz};
  }
  // replaces the active shape's point shell (analytic SDF kept)
  void setShellPoints(const std::vector<R>& p) {
    const int n = (int)(p.size() / 3);
    shell.assign(n > 0 ? n : 1, V3<R>{0, 0, 0});
    for (int i = 0; i < n; ++i)
      shell[i] = V3<R>{p[3 * i], p[3 * i + 1], p[3 * i + 2]};
    shapes[0].numPoints = n;
    shapes[0].shellOffset = 0;
    shellPoints = n;
    ensureContactCapacity();
  }
  // sim.hpp:1034-1084
  void setSdfShape(const std::vector<R>& grid, int nx, int ny, int nz, V3<R> origin, V3<R> spacing,
                   const std::vector<R>& shellFlat, V3<R> invIn, R boundingRadius) {
    if (nx < 2 || ny < 2 || nz < 2)
      throw std::runtime_error("setSdfShape: grid dims must be >= 2 on each axis");
    if ((long)nx * ny * nz != (long)grid.size())
      throw std::runtime_error("setSdfShape: grid.size() must equal nx*ny*nz");
    const int n = (int)(shellFlat.size() / 3);
    if (n <= 0)
      throw std::runtime_error("setSdfShape: empty surface point shell");
    sdfGrid = grid;
    shell.resize(n);
    for (int i = 0; i < n; ++i)
      shell[i] = V3<R>{shellFlat[3 * i], shellFlat[3 * i + 1], shellFlat[3 * i + 2]};
    Shape<R> d;
    d.type = GRID;
    d.par = V4<R>{boundingRadius, 0, 0, 0};
    d.numPoints = n;
    d.nx = nx;
    d.ny = ny;
    d.nz = nz;
    d.gridOrigin = origin;
    d.gridInvSpacing = V3<R>{spacing.x > 0 ? R(1) / spacing.x : R(0), spacing.y > 0 ? R(1) / spacing.y : R(0),
                             spacing.z > 0 ? R(1) / spacing.z : R(0)};
    shapes[0] = d;
    baseRadius = boundingRadius;
    defaultInvI = invIn;
    shellPoints = n;
    ensureContactCapacity();
  }
  void setDomain(R lx, R ly, R lz, bool ppx, bool ppy, bool ppz) {  // sim.hpp:1086-1089
    dmin = V3<R>{0, 0, 0};
    dmax = V3<R>{lx, ly, lz};
    dsize = V3<R>{lx, ly, lz};
    px = ppx;
    py = ppy;
    pz = ppz;
    skin = R(0.1) * globalScale;
  }
  void setDomainMinMax(V3<R> mn, V3<R> mx) {  // sim.hpp:1091-1099
    dmin = mn;
    dmax = mx;
    dsize = sub(mx, mn);
    skin = R(0.1) * globalScale;
  }
  void setPairMaterial(int a, int b, R e, R f) {  // sim.hpp:1196-1216
    if (a < 0 || b < 0 || a >= kMaxMaterials || b >= kMaxMaterials)
      throw std::invalid_argument("material id out of range");
    if (pairMat.empty()) {
      pairMat.assign(kMaxMaterials * kMaxMaterials * 2, R(0));
      for (int i = 0; i < kMaxMaterials * kMaxMaterials; ++i) {
        pairMat[2 * i] = eN;
        pairMat[2 * i + 1] = mu;
      }
    }
    pairMat[(a * kMaxMaterials + b) * 2] = e;
    pairMat[(a * kMaxMaterials + b) * 2 + 1] = f;
    pairMat[(b * kMaxMaterials + a) * 2] = e;
    pairMat[(b * kMaxMaterials + a) * 2 + 1] = f;
  }
  void addPlane(V3<R> p, V3<R> n) {  // sim.hpp:1226-1232
    if ((int)planes.size() < planeCap)
      planes.push_back(Plane<R>{p, n});
  }
  int addSdfWall(const std::vector<R>& grid, int nx, int ny, int nz, V3<R> origin, V3<R> spacing,
                 R e, R f) {  // sim.hpp:1242-1274
    if (nx < 2 || ny < 2 || nz < 2)
      throw std::runtime_error("addSdfWall: grid dims must be >= 2 on each axis");
    if ((long)nx * ny * nz != (long)grid.size())
      throw std::runtime_error("addSdfWall: grid.size() must equal nx*ny*nz");
    Wall<R> w;
    w.nx = nx;
    w.ny = ny;
    w.nz = nz;
    const bool first = walls.empty();
    w.gridOffset = first ? 0 : (int)wallGrid.size();
    w.origin = origin;
    w.invSpacing = V3<R>{spacing.x > 0 ? R(1) / spacing.x : R(0), spacing.y > 0 ? R(1) / spacing.y : R(0),
                         spacing.z > 0 ? R(1) / spacing.z : R(0)};
    w.restitution = e;
    w.friction = f;
    if (first)
      wallGrid.clear();
    wallGrid.insert(wallGrid.end(), grid.begin(), grid.end());
    walls.push_back(w);
    if (f > wallFrictionMax)
      wallFrictionMax = f;
    ensureContactCapacity();
    return (int)walls.size() - 1;
  }
  void setPositions(const std::vector<R>& xyz) {  // sim.hpp:1290-1330
    const int n = (int)(xyz.size() / 3);
    numReal = n;
    numParticles = n;
    hzNumPairs = -1;
    hzPrevCount = 0;
    for (int i = 0; i < n; ++i) {
      pos[i] = V3<R>{xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
      quat[i] = V4<R>{0, 0, 0, 1};
      invMass[i] = 1;
      scale[i] = 1;
      shapeId[i] = 0;
      invI[i] = defaultInvI;
      vel[i] = V3<R>{0, 0, 0};
      angVel[i] = V3<R>{0, 0, 0};
    }
    for (int i = 0; i < capacity; ++i)
      targetScale[i] = scale[i];
  }

  // ---------------- integration (src/integration.hpp) ----------------
  // integration.hpp:44-93
  void predictVelocity(int n) {
    const R dtt = dt;
    for (int i = 0; i < n; ++i) {
      const R im = invMass[i];
      V3<R> v = vel[i];
      if (im > R(0)) {
        v = add(v, mul(gravity, dtt));
        v = add(v, mul(extForce[i], im * dtt));
      }
      velPred[i] = v;
      V3<R> wp = angVel[i];
      if (im > R(0)) {
        const V3<R> ii = invI[i];
        if (ii.x > R(0) || ii.y > R(0) || ii.z > R(0)) {
          const V4<R> q = quat[i];
          V3<R> wb = invrot(q, angVel[i]);
          const V3<R> Ib{(ii.x > R(1e-9)) ? R(1) / ii.x : R(0), (ii.y > R(1e-9)) ? R(1) / ii.y : R(0),
                         (ii.z > R(1e-9)) ? R(1) / ii.z : R(0)};
          const V3<R> Lb{Ib.x * wb.x, Ib.y * wb.y, Ib.z * wb.z};
          const V3<R> wxL = cross(wb, Lb);
          const V3<R> al{-ii.x * wxL.x, -ii.y * wxL.y, -ii.z * wxL.z};
          wb = add(wb, mul(al, dtt));
          wp = rot(q, wb);
        }
      }
      angVelPred[i] = wp;
      V3<R> x = pos[i];
      if (im > R(0))
        x = add(x, mul(v, dtt));
      posPred[i] = x;
      quatPred[i] = quat[i];
      deltaVel[i] = deltaAngVel[i] = deltaPos[i] = V3<R>{0, 0, 0};
      constraintCounts[i] = 0;
    }
  }
  // integration.hpp:97-109
  void applyVelocityDeltas(int n) {
    for (int i = 0; i < n; ++i) {
      velPred[i] = add(velPred[i], deltaVel[i]);
      angVelPred[i] = add(angVelPred[i], deltaAngVel[i]);
      deltaVel[i] = deltaAngVel[i] = V3<R>{0, 0, 0};
    }
  }
  // integration.hpp:112-148
  void applyVelocityAndPredictPosition(int n) {
    const R dtt = dt;
    for (int i = 0; i < n; ++i) {
      const V3<R> vs = vel[i];
      const V3<R> vf = velPred[i];
      velPred[i] = vf;
      vel[i] = vf;
      const R im = invMass[i];
      V3<R> x = pos[i];
      if (im > R(0))
        x = add(x, mul(add(vs, vf), R(0.5) * dtt));
      posPred[i] = x;
      const V4<R> q = quat[i];
      const V3<R> w = angVelPred[i];
      angVel[i] = w;
      V4<R> qp = q;
      if (im > R(0)) {
        qp.x += R(0.5) * dtt * (w.x * q.w + w.y * q.z - w.z * q.y);
        qp.y += R(0.5) * dtt * (w.y * q.w + w.z * q.x - w.x * q.z);
        qp.z += R(0.5) * dtt * (w.z * q.w + w.x * q.y - w.y * q.x);
        qp.w += R(0.5) * dtt * (-w.x * q.x - w.y * q.y - w.z * q.z);
        const R l = std::sqrt(qp.x * qp.x + qp.y * qp.y + qp.z * qp.z + qp.w * qp.w);
        if (l > R(1e-9)) {
          const R s = R(1) / l;
          qp = V4<R>{qp.x * s, qp.y * s, qp.z * s, qp.w * s};
        }
      }
      quatPred[i] = qp;
    }
  }
  // integration.hpp:168-184
  void applyUpdates(int n) {
    for (int i = 0; i < n; ++i) {
      const int c = constraintCounts[i];
      if (c <= 0)
        continue;
      const R f = R(1) / static_cast<R>(c);
      posPred[i] = add(posPred[i], mul(deltaPos[i], f));
      velPred[i] = add(velPred[i], mul(deltaVel[i], f));
      deltaPos[i] = deltaVel[i] = V3<R>{0, 0, 0};
      constraintCounts[i] = 0;
    }
  }
  // integration.hpp:187-215
  void finalCommit(int n) {
    for (int i = 0; i < n; ++i) {
      V3<R> p = posPred[i];
      if (px) {
        if (p.x < dmin.x)
          p.x += dsize.x;
        else if (p.x >= dmax.x)
          p.x -= dsize.x;
      }
      if (py) {
        if (p.y < dmin.y)
          p.y += dsize.y;
        else if (p.y >= dmax.y)
          p.y -= dsize.y;
      }
      if (pz) {
        if (p.z < dmin.z)
          p.z += dsize.z;
        else if (p.z >= dmax.z)
          p.z -= dsize.z;
      }
      pos[i] = p;
      quat[i] = quatPred[i];
    }
  }
  // integration.hpp:229-272 (kinetic energies summed in double, ascending index)
  void thermostat(int n) {
    double kt = 0.0, kr = 0.0;
    for (int i = 0; i < n; ++i) {
      const R im = invMass[i];
      const V3<R> v = vel[i];
      if (im > R(0))
        kt += 0.5 * (1.0 / (double)im) * (double)(v.x * v.x + v.y * v.y + v.z * v.z);
      const V3<R> ii = invI[i];
      if (ii.x > R(0) || ii.y > R(0) || ii.z > R(0)) {
        const V3<R> wb = invrot(quat[i], angVel[i]);
        const double Ix = (ii.x > R(0)) ? 1.0 / (double)ii.x : 0.0;
        const double Iy = (ii.y > R(0)) ? 1.0 / (double)ii.y : 0.0;
        const double Iz = (ii.z > R(0)) ? 1.0 / (double)ii.z : 0.0;
        kr += 0.5 * (Ix * (double)wb.x * (double)wb.x + Iy * (double)wb.y * (double)wb.y +
                      Iz * (double)wb.z * (double)wb.z);
      }
    }
    const double ndof = 3.0 * n;
    const double kB = (double)thermoKB, tau = (double)thermoTau, Tt = (double)thermoTemp;
    auto lam = [&](double ke) -> R {
      if (ndof <= 0 || kB <= 0)
        return R(1);
      const double Tc = (2.0 * ke) / (ndof * kB);
      if (Tc < 1e-6)
        return R(1);
      double f = 1.0 + ((double)dt / tau) * (Tt / Tc - 1.0);
      if (f < 0.0)
        f = 0.0;
      return static_cast<R>(std::sqrt(f));
    };
    const R lt = lam(kt), lr = lam(kr);
    for (int i = 0; i < n; ++i) {
      vel[i] = mul(vel[i], lt);
      angVel[i] = mul(angVel[i], lr);
    }
  }
  // integration.hpp:275-283
  void updateGrowthScales(int n, R factor) {
    if (!(factor > R(0)))
      return;
    for (int i = 0; i < n; ++i)
      scale[i] = targetScale[i] * factor;
  }

  // ---------------- ghosts (src/periodicity.hpp) ----------------
  // periodicity.hpp:25-38
  int ghostCapacity(int nReal, R skinW) const {
    const R sx = px ? skinW : R(0), sy = py ? skinW : R(0), sz = pz ? skinW : R(0);
    const double ix = (dsize.x - R(2) * sx > R(0)) ? (double)(dsize.x - R(2) * sx) : 0.0;
    const double iy = (dsize.y - R(2) * sy > R(0)) ? (double)(dsize.y - R(2) * sy) : 0.0;
    const double iz = (dsize.z - R(2) * sz > R(0)) ? (double)(dsize.z - R(2) * sz) : 0.0;
    const double vt = (double)dsize.x * (double)dsize.y * (double)dsize.z;
    if (vt <= 0.0)
      return nReal * 8;
    const double gf = (vt - ix * iy * iz) / vt;
    const double est = (gf > 0.5) ? nReal * 32.0 : nReal * gf * 4.0;
    return nReal + (int)est + 4096;
  }
  // periodicity.hpp:43-94 (slots in ascending (particle, image) order; overflow dropped)
  void generateGhosts(R skinW) {
    for (int i = 0; i < numReal; ++i) {
      const V3<R> p = pos[i];
      const int sx = px ? ((p.x < dmin.x + skinW) ? 1 : ((p.x > dmax.x - skinW) ? -1 : 0)) : 0;
      const int sy = py ? ((p.y < dmin.y + skinW) ? 1 : ((p.y > dmax.y - skinW) ? -1 : 0)) : 0;
      const int sz = pz ? ((p.z < dmin.z + skinW) ? 1 : ((p.z > dmax.z - skinW) ? -1 : 0)) : 0;
      const int ax[2] = {0, sx}, ay[2] = {0, sy}, az[2] = {0, sz};
      const int nx = sx == 0 ? 1 : 2, ny = sy == 0 ? 1 : 2, nz = sz == 0 ? 1 : 2;
      const V3<R> pp = posPred[i];
      for (int a = 0; a < nx; ++a)
        for (int b = 0; b < ny; ++b)
          for (int c = 0; c < nz; ++c) {
            const int ix = ax[a], iy = ay[b], iz = az[c];
            if (ix == 0 && iy == 0 && iz == 0)
              continue;
            const int slot = topGhost;
            if (slot >= capacity)
              continue;
            ++topGhost;
            const V3<R> sh{ix * dsize.x, iy * dsize.y, iz * dsize.z};
            pos[slot] = add(p, sh);
            posPred[slot] = add(pp, sh);
            invMass[slot] = invMass[i];
            vel[slot] = vel[i];
            velPred[slot] = velPred[i];
            quat[slot] = quat[i];
            quatPred[slot] = quatPred[i];
            angVel[slot] = angVel[i];
            angVelPred[slot] = angVelPred[i];
            scale[slot] = scale[i];
            shapeId[slot] = shapeId[i];
            realIdx[slot] = i;
          }
    }
  }

  // ---------------- broadphase (src/broadphase_arborx.hpp:36-107, src/sim.hpp:82-94) ----------
  struct Box {
    R lo[3], hi[3];
  };
  Box saneBox(int i, const std::vector<V3<R>>& P, R margin, R boxCap) const {
    R x = P[i].x, y = P[i].y, z = P[i].z, b = rad[i] + margin;
    if (!(b == b) || !(x == x) || !(y == y) || !(z == z) || (boxCap > R(0) && b > boxCap)) {
      x = y = z = R(-1.0e30);
      b = 0;
    }
    return Box{{x - b, y - b, z - b}, {x + b, y + b, z + b}};
  }
  static bool overlap(const Box& a, const Box& b) {
    for (int d = 0; d < 3; ++d)
      if (a.lo[d] > b.hi[d] || a.hi[d] < b.lo[d])
        return false;
    return true;
  }
  // Exact candidate set of the reference query (closed-box corner overlap), emitted sorted by
  // (i, j), i real, j > i. A sort-and-sweep on the lower x corner makes it O(N log N + P).
  int findCollisions(const std::vector<V3<R>>& P, R margin, std::vector<int>& out) {
    const R boxCap = std::max(std::max(dsize.x, dsize.y), dsize.z);
    const int n = numParticles;
    std::vector<Box> bx(n);
    for (int i = 0; i < n; ++i)
      bx[i] = saneBox(i, P, margin, boxCap);
    std::vector<int> ord(n);
    std::iota(ord.begin(), ord.end(), 0);
    std::sort(ord.begin(), ord.end(), [&](int a, int b) {
      return bx[a].lo[0] < bx[b].lo[0] || (bx[a].lo[0] == bx[b].lo[0] && a < b);
    });
    std::vector<R> los(n);
    for (int t = 0; t < n; ++t)
      los[t] = bx[ord[t]].lo[0];
    std::vector<int> hit;
    out.clear();
    for (int i = 0; i < numReal; ++i) {
      hit.clear();
      // candidates: lo.x <= hi_i.x; and hi.x >= lo_i.x checked exactly
      const int end = (int)(std::upper_bound(los.begin(), los.end(), bx[i].hi[0]) - los.begin());
      for (int t = 0; t < end; ++t) {
        const int j = ord[t];
        if (j > i && overlap(bx[i], bx[j]))
          hit.push_back(j);
      }
      std::sort(hit.begin(), hit.end());
      for (int j : hit) {
        out.push_back(i);
        out.push_back(j);
      }
    }
    return (int)(out.size() / 2);
  }
  int findCollisionsGrow(R margin) {
    std::vector<int> all;
    const int np = findCollisions(posPred, margin, all);
    if (np > maxPairs) {
      maxPairs = np + np / 2 + 64;
      pairs.assign(2 * (size_t)maxPairs, 0);
    }
    std::copy(all.begin(), all.end(), pairs.begin());
    pairCount = np;
    return std::min(np, maxPairs);
  }

  // ---------------- narrowphase (src/narrowphase.hpp) ----------------
  bool pushContact(const Contact<R>& c) {
    if (contactCount >= maxContacts)
      return false;
    contacts[contactCount++] = c;
    return true;
  }
  // narrowphase.hpp:179-268
  void detectContacts(int np, R margin) {
    for (int idx = 0; idx < np; ++idx) {
      const int A = pairs[2 * idx], B = pairs[2 * idx + 1];
      const Shape<R>& dA = shapes[shapeId[A]];
      const Shape<R>& dB = shapes[shapeId[B]];
      const V3<R> pA = posPred[A], pB = posPred[B];
      const V4<R> qA = quatPred[A], qB = quatPred[B];
      const R sA = scale[A] * globalScale, sB = scale[B] * globalScale;
      const int cnt = dA.numPoints;
      const bool sphA = dA.type == SPHERE;
      const int iter = cnt > 0 ? cnt : 1;
      for (int k = 0; k < iter; ++k) {
        V3<R> pl{0, 0, 0};
        R prad = 0;
        if (cnt > 0)
          pl = shell[dA.shellOffset + k];
        else if (sphA)
          prad = dA.par.x * sA;
        const V3<R> pw = add(pA, rot(qA, mul(pl, sA)));
        const V3<R> plB = invrot(qB, sub(pw, pB));
        const V3<R> pc = mul(plB, R(1) / sB);
        const R dist = sdfShape(pc, dB, sdfGrid.data()) * sB;
        const R eff = dist - prad;
        if (eff >= margin)
          continue;
        if (eff < R(0))
          maxOverlap = std::max(maxOverlap, -eff);
        if (contactCount >= maxContacts)
          continue;
        const R eps = R(1e-4);
        V3<R> nl{sdfShape(V3<R>{pc.x + eps, pc.y, pc.z}, dB, sdfGrid.data()) -
                     sdfShape(V3<R>{pc.x - eps, pc.y, pc.z}, dB, sdfGrid.data()),
                 sdfShape(V3<R>{pc.x, pc.y + eps, pc.z}, dB, sdfGrid.data()) -
                     sdfShape(V3<R>{pc.x, pc.y - eps, pc.z}, dB, sdfGrid.data()),
                 sdfShape(V3<R>{pc.x, pc.y, pc.z + eps}, dB, sdfGrid.data()) -
                     sdfShape(V3<R>{pc.x, pc.y, pc.z - eps}, dB, sdfGrid.data())};
        const R l = len(nl);
        nl = (l > R(1e-9)) ? mul(nl, R(1) / l) : V3<R>{0, 1, 0};
        const V3<R> nw = rot(qB, nl);
        const V3<R> ps = sub(pw, mul(nw, prad));
        Contact<R> c;
        c.a = A;
        c.b = B;
        c.n = nw;
        c.rA = sub(ps, pA);
        c.rB = sub(sub(ps, mul(nw, eff)), pB);
        c.dist = eff;
        if (!pairMat.empty()) {
          const int t = (int(materialId[A]) * kMaxMaterials + int(materialId[B])) * 2;
          c.e = pairMat[t];
          c.mu = pairMat[t + 1];
        }
        pushContact(c);
      }
    }
  }
  // narrowphase.hpp:371-449
  void detectBoundary(R margin) {
    for (int i = 0; i < numReal; ++i) {
      const V3<R> pA = posPred[i];
      const R s = scale[i] * globalScale;
      const Shape<R>& d = shapes[shapeId[i]];
      R bR = d.par.x;
      if (bR == R(0))
        bR = 1;
      const R radius = bR * s;
      const int npts = d.numPoints;
      const V4<R> qA = quatPred[i];
      for (const Plane<R>& pl : planes) {
        if (npts > 0) {
          for (int k = 0; k < npts; ++k) {
            const V3<R> rA = rot(qA, mul(shell[d.shellOffset + k], s));
            const V3<R> pw = add(pA, rA);
            const R dist = dot(sub(pw, pl.p), pl.n);
            if (dist >= margin)
              continue;
            if (dist < R(0))
              maxOverlap = std::max(maxOverlap, -dist);
            Contact<R> c;
            c.a = i;
            c.b = -1;
            c.n = pl.n;
            c.rA = rA;
            c.rB = pl.p;
            c.dist = dist;
            pushContact(c);
          }
        } else {
          const R dist = dot(sub(pA, pl.p), pl.n) - radius;
          if (dist >= margin)
            continue;
          if (dist < R(0))
            maxOverlap = std::max(maxOverlap, -dist);
          Contact<R> c;
          c.a = i;
          c.b = -1;
          c.n = pl.n;
          c.rA = mul(pl.n, -radius);
          c.rB = pl.p;
          c.dist = dist;
          pushContact(c);
        }
      }
    }
  }
  // narrowphase.hpp:278-367
  void detectWallSdf(R margin) {
    const R* g = wallGrid.data();
    for (int i = 0; i < numReal; ++i) {
      const V3<R> pA = posPred[i];
      const R s = scale[i] * globalScale;
      const Shape<R>& d = shapes[shapeId[i]];
      R bR = d.par.x;
      if (bR == R(0))
        bR = 1;
      const R radius = bR * s;
      const int npts = d.numPoints;
      const V4<R> qA = quatPred[i];
      const R eps = R(1e-4);
      for (const Wall<R>& w : walls) {
        const int iter = npts > 0 ? npts : 1;
        for (int k = 0; k < iter; ++k) {
          V3<R> rA{0, 0, 0};
          if (npts > 0)
            rA = rot(qA, mul(shell[d.shellOffset + k], s));
          const V3<R> pw = add(pA, rA);
          const R sdf = sampleWall(pw, w, g);
          V3<R> n{sampleWall(V3<R>{pw.x + eps, pw.y, pw.z}, w, g) - sampleWall(V3<R>{pw.x - eps, pw.y, pw.z}, w, g),
                  sampleWall(V3<R>{pw.x, pw.y + eps, pw.z}, w, g) - sampleWall(V3<R>{pw.x, pw.y - eps, pw.z}, w, g),
                  sampleWall(V3<R>{pw.x, pw.y, pw.z + eps}, w, g) - sampleWall(V3<R>{pw.x, pw.y, pw.z - eps}, w, g)};
          const R ln = len(n);
          n = (ln > R(1e-9)) ? mul(n, R(1) / ln) : V3<R>{0, 1, 0};
          const R dist = (npts > 0) ? sdf : sdf - radius;
          if (dist >= margin)
            continue;
          const V3<R> rAe = (npts > 0) ? rA : mul(n, -radius);
          const V3<R> ps = add(pA, rAe);
          const V3<R> pWall = sub(ps, mul(n, dist));
          if (dist < R(0))
            maxOverlap = std::max(maxOverlap, -dist);
          if (contactCount >= maxContacts)
            continue;
          const V3<R> vW = add(w.linVel, cross(w.angVel, sub(pWall, w.center)));
          Contact<R> c;
          c.a = i;
          c.b = -1;
          c.n = n;
          c.rA = rAe;
          c.rB = pWall;
          c.dist = dist;
          c.bvel = vW;
          if (w.materialId >= 0 && !pairMat.empty()) {
            const int t = (int(materialId[i]) * kMaxMaterials + w.materialId) * 2;
            c.e = pairMat[t];
            c.mu = pairMat[t + 1];
          } else {
            c.e = w.restitution;
            c.mu = w.friction;
          }
          pushContact(c);
        }
      }
    }
  }

  // ---------------- contact -> manifold (src/contact_preprocessing.hpp:320-471) ---------------
  static u64 contactKey(const Contact<R>& c) {  // :320-327
    if (c.b < 0)
      return ((u64)(unsigned)c.a << 32) | 0xFFFFFFFFull;
    const unsigned u = c.a < c.b ? c.a : c.b, v = c.a < c.b ? c.b : c.a;
    return ((u64)u << 32) | v;
  }
  static Manifold<R> toManifold(const Contact<R>& c) {  // :339-374
    Manifold<R> m;
    if (c.dist > R(0)) {
      m.np = 0;
      m.e = 0;
      m.mu = 0;
      return m;
    }
    const bool flip = (c.b >= 0 && c.b < c.a);
    m.np = 1;
    const V3<R> na = flip ? c.n : neg(c.n);
    const V3<R> sh{c.n.x * c.dist * R(0.5), c.n.y * c.dist * R(0.5), c.n.z * c.dist * R(0.5)};
    const V3<R> ra = sub(c.rA, sh);
    const V3<R> rb = add(c.rB, sh);
    const V3<R> rc = flip ? rb : ra, ro = flip ? ra : rb;
    m.N = na;
    m.TA = cross(rc, na);
    m.TB = cross(ro, neg(na));
    m.rA = rc;
    m.rB = ro;
    m.wv = c.bvel;
    m.e = c.e;
    m.mu = c.mu;
    return m;
  }
  int reduceToManifolds(int n) {  // :378-471
    if (n == 0) {
      manifoldCount = 0;
      return 0;
    }
    std::vector<u64> keys(n);
    std::vector<int> perm(n);
    for (int i = 0; i < n; ++i) {
      keys[i] = contactKey(contacts[i]);
      perm[i] = i;
    }
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return keys[a] < keys[b]; });
    int nseg = 0;
    for (int p = 0; p < n; ++p) {
      const u64 k = keys[perm[p]];
      const bool lead = p == 0 || k != keys[perm[p - 1]];
      if (lead) {
        Manifold<R> m;
        m.a = (int)(k >> 32);
        const unsigned v = (unsigned)(k & 0xFFFFFFFFull);
        m.b = v == 0xFFFFFFFFu ? -1 : (int)v;
        manifolds[nseg++] = m;
      }
      const Manifold<R> t = toManifold(contacts[perm[p]]);
      Manifold<R>& o = manifolds[nseg - 1];
      o.np += t.np;
      o.N = add(o.N, t.N);
      o.TA = add(o.TA, t.TA);
      o.TB = add(o.TB, t.TB);
      o.rA = add(o.rA, t.rA);
      o.rB = add(o.rB, t.rB);
      o.wv = add(o.wv, t.wv);
      o.e += t.e;
      o.mu += t.mu;
      contactSlot[perm[p]] = nseg - 1;
    }
    manifoldCount = nseg;
    return nseg;
  }

  // ---------------- warm-start ledger (src/contact_preprocessing.hpp:70-253) ----------------
  u64 keyOf(const Manifold<R>& m) const {  // :70-76
    const unsigned a = (unsigned)realIdx[m.a];
    const unsigned b = m.b >= 0 ? (unsigned)realIdx[m.b] : 0xFFFFFFFFu;
    const unsigned hi = a < b ? a : b, lo = a < b ? b : a;
    return ((u64)hi << 32) | lo;
  }
  int lowerBound(const std::vector<u64>& keys, int n, u64 k) const {
    int lo = 0, hi = n;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (keys[mid] < k)
        lo = mid + 1;
      else
        hi = mid;
    }
    return lo;
  }
  void gatherWarm(int nm) {  // :113-156
    for (int i = 0; i < nm; ++i) {
      const Manifold<R>& m = manifolds[i];
      const bool dup = m.np > 0 && m.b >= 0 && realIdx[m.a] > realIdx[m.b];
      if (m.np <= 0 || dup) {
        pairKeys[i] = ~0ull;
        lambdaAcc[i] = 0;
        lambdaT[i] = V3<R>{0, 0, 0};
        posImpulse[i] = 0;
        continue;
      }
      const u64 k = keyOf(m);
      pairKeys[i] = k;
      const int lo = lowerBound(prevPairKeys, prevPairCount, k);
      const bool hit = lo < prevPairCount && prevPairKeys[lo] == k;
      lambdaAcc[i] = hit ? prevLambda[lo] : R(0);
      lambdaT[i] = hit ? prevLambdaT[lo] : V3<R>{0, 0, 0};
      posImpulse[i] = hit ? prevPosImpulse[lo] : R(0);
    }
  }
  void markPersistent(int nm) {  // :78-108
    for (int i = 0; i < nm; ++i) {
      const Manifold<R>& m = manifolds[i];
      if (m.np <= 0) {
        pairKeys[i] = ~0ull;
        persistent[i] = 0;
        continue;
      }
      const u64 k = keyOf(m);
      pairKeys[i] = k;
      const int lo = lowerBound(prevPairKeys, prevPairCount, k);
      persistent[i] = (lo < prevPairCount && prevPairKeys[lo] == k) ? 1 : 0;
    }
  }
  void updateGrounded(int nm, V3<R> gHat, int sweeps, int decay) {  // :213-253
    for (int i = 0; i < numReal; ++i) {
      const int g = (int)grounded[i] - decay;
      grounded[i] = (unsigned char)(g > 0 ? g : 0);
    }
    for (int s = 0; s < sweeps; ++s)
      for (int i = 0; i < nm; ++i) {
        const Manifold<R>& m = manifolds[i];
        if (m.np <= 0)
          continue;
        const int ra = realIdx[m.a];
        if (m.b < 0) {
          grounded[ra] = 255;
          continue;
        }
        const int rb = realIdx[m.b];
        const V3<R> dx = sub(posPred[m.a], posPred[m.b]);
        const R up = -(dx.x * gHat.x + dx.y * gHat.y + dx.z * gHat.z);
        const R thr = R(0.3) * std::sqrt(dot(dx, dx));
        if (up > thr) {
          const int l = (int)grounded[rb] - 1;
          if (l > 0 && (unsigned char)l > grounded[ra])
            grounded[ra] = (unsigned char)l;
        } else if (up < -thr) {
          const int l = (int)grounded[ra] - 1;
          if (l > 0 && (unsigned char)l > grounded[rb])
            grounded[rb] = (unsigned char)l;
        }
      }
  }
  // height-from-floor levels of the "ordered" pass (contact_preprocessing.hpp:263-305): 0 at a
  // wall or plane contact, else 1 + min over supporting bodies, relaxed to a fixed point
  static constexpr int kLevelInf = 1 << 28;
  std::vector<int> heightLevel;
  void computeHeightLevels(int nm, V3<R> gHat) {
    heightLevel.assign(numReal, kLevelInf);
    for (int s = 0; s < 1024; ++s) {
      int changed = 0;
      for (int i = 0; i < nm; ++i) {
        const Manifold<R>& m = manifolds[i];
        if (m.np <= 0)
          continue;
        const int ra = realIdx[m.a];
        if (m.b < 0) {
          if (heightLevel[ra] > 0) {
            heightLevel[ra] = 0;
            ++changed;
          }
          continue;
        }
        const int rb = realIdx[m.b];
        const V3<R> dx = sub(posPred[m.a], posPred[m.b]);
        const R up = -(dx.x * gHat.x + dx.y * gHat.y + dx.z * gHat.z);
        const R thr = R(0.3) * std::sqrt(dot(dx, dx));
        if (up > thr) {
          const int cand = heightLevel[rb];
          if (cand < kLevelInf && heightLevel[ra] > cand + 1) {
            heightLevel[ra] = cand + 1;
            ++changed;
          }
        } else if (up < -thr) {
          const int cand = heightLevel[ra];
          if (cand < kLevelInf && heightLevel[rb] > cand + 1) {
            heightLevel[rb] = cand + 1;
            ++changed;
          }
        }
      }
      if (changed == 0)
        break;
    }
  }
  // level-ordered symmetric sweeps (solver_velocity.hpp:914-989; sim.hpp:357-400): the coloured
  // manifolds bucketed by (level, colour), key level * 64 + colour (stable), swept bottom-up then
  // top-down per iteration until the residual drains
  // ---------------- multilevel stabilization (src/sim.hpp:303-356, src/solver_multilevel.hpp) ----------------
  // Greedy pairwise aggregation of the quasi-static contact graph into super-bodies, per level a
  // colouring of the manifolds that cross aggregate boundaries; per iteration one fine PGS sweep,
  // then on every level a restriction (momentum-weighted group velocity), two translation-only
  // coarse PGS sweeps at the aggregate masses on the shared normal accumulator, and a
  // prolongation; the loop stops on the quasi-static residual.
  static constexpr int kMlMaxLevels = 10, kMlSkip = 63, kMlGateSlip = 4;
  std::vector<long long> mlPacked;
  std::vector<int> mlParent, mlGrp, mlMate;
  std::vector<R> mlMassG, mlInvMassG;
  std::vector<V3<R>> mlVelG, mlVelG0;
  struct MlLevel {
    int groupOff, numGroups, parentOff, numColors;
  };
  static R mlEffMass(R im) { return R(1) / std::fmax(im, R(1e-30)); }  // solver_multilevel.hpp:79-81
  bool mlEligible(int idx, R qsThr) const {  // solver_multilevel.hpp:97-128, gates = slip
    const Manifold<R>& m = manifolds[idx];
    if (m.np <= 0 || mColor[idx] < 0)
      return false;
    if (std::fabs(vn0[idx]) > qsThr)
      return false;
    if (dot(vt0[idx], vt0[idx]) > qsThr * qsThr)
      return false;
    return true;
  }
  std::vector<MlLevel> mlBuild(int nm, R qsThr) {  // solver_multilevel.hpp:134-323
    std::vector<MlLevel> H;
    if (nm <= 0 || numReal <= 0)
      return H;
    mlPacked.assign(nm, ~0ll);
    mlGrp.resize(numReal);
    for (int i = 0; i < numReal; ++i)
      mlGrp[i] = i;
    const int parentCap = 5 * capacity, groupCap = 4 * capacity;
    mlParent.resize(parentCap);
    mlMassG.resize(groupCap);
    mlInvMassG.resize(groupCap);
    mlVelG.resize(groupCap);
    mlVelG0.resize(groupCap);
    mlMate.resize(std::max(numReal, 1));
    std::vector<long long> winner(std::max(numReal, 1));
    std::vector<u64> mask(std::max(numReal, 1));
    int ngPrev = numReal, parentOff = 0, groupOff = 0;
    for (int lvl = 1; lvl <= kMlMaxLevels; ++lvl) {
      if (parentOff + ngPrev > parentCap)
        break;
      for (int g = 0; g < ngPrev; ++g)
        winner[g] = -1;
      auto ends = [&](int idx, int& gA, int& gB) {
        const Manifold<R>& m = manifolds[idx];
        gA = mlGrp[realIdx[m.a]];
        gB = m.b >= 0 ? mlGrp[realIdx[m.b]] : -1;
      };
      for (int idx = 0; idx < nm; ++idx) {  // matching: contend
        if (manifolds[idx].b < 0 || !mlEligible(idx, qsThr))
          continue;
        int gA, gB;
        ends(idx, gA, gB);
        if (gA == gB)
          continue;
        const long long key = colorKey(idx);
        winner[gA] = std::max(winner[gA], key);
        winner[gB] = std::max(winner[gB], key);
      }
      for (int g = 0; g < ngPrev; ++g)
        mlMate[g] = g;
      for (int idx = 0; idx < nm; ++idx) {  // matching: sole winner of both ends
        if (manifolds[idx].b < 0 || !mlEligible(idx, qsThr))
          continue;
        int gA, gB;
        ends(idx, gA, gB);
        if (gA == gB)
          continue;
        const long long key = colorKey(idx);
        if (winner[gA] == key && winner[gB] == key) {
          mlMate[gA] = gB;
          mlMate[gB] = gA;
        }
      }
      int ngNew = 0;  // compaction: a matched pair -> one id (leader = the smaller)
      for (int g = 0; g < ngPrev; ++g)
        if (mlMate[g] >= g)
          mlParent[parentOff + g] = ngNew++;
      for (int g = 0; g < ngPrev; ++g)
        if (mlMate[g] < g)
          mlParent[parentOff + g] = mlParent[parentOff + mlMate[g]];
      if (ngNew >= ngPrev || ngNew > (9 * ngPrev) / 10)
        break;
      if (groupOff + ngNew > groupCap)
        break;
      for (int i = 0; i < numReal; ++i)
        mlGrp[i] = mlParent[parentOff + mlGrp[i]];
      for (int g = 0; g < ngNew; ++g)
        mlMassG[groupOff + g] = 0;
      for (int i = 0; i < numReal; ++i)
        mlMassG[groupOff + mlGrp[i]] += mlEffMass(invMass[i]);
      for (int g = 0; g < ngNew; ++g)
        mlInvMassG[groupOff + g] = R(1) / mlMassG[groupOff + g];
      // colouring of the crossing manifolds on the group graph (this level's 6-bit slot)
      const int shift = 6 * (lvl - 1);
      for (int g = 0; g < ngNew; ++g)
        mask[g] = 0;
      int remaining = 1, prevRemaining = -1, maxc = -1;
      for (int round = 0; round < 64 && remaining > 0; ++round) {
        for (int g = 0; g < ngNew; ++g)
          winner[g] = -1;
        auto pending = [&](int idx, int& gA, int& gB) {
          if (!mlEligible(idx, qsThr) || ((mlPacked[idx] >> shift) & 63) != kMlSkip)
            return false;
          ends(idx, gA, gB);
          return gB != gA;
        };
        for (int idx = 0; idx < nm; ++idx) {
          int gA, gB;
          if (!pending(idx, gA, gB))
            continue;
          const long long key = colorKey(idx);
          winner[gA] = std::max(winner[gA], key);
          if (gB >= 0)
            winner[gB] = std::max(winner[gB], key);
        }
        int rem = 0;
        for (int idx = 0; idx < nm; ++idx) {
          int gA, gB;
          if (!pending(idx, gA, gB))
            continue;
          const long long key = colorKey(idx);
          if (winner[gA] != key || (gB >= 0 && winner[gB] != key)) {
            ++rem;
            continue;
          }
          u64 forb = mask[gA] | (gB >= 0 ? mask[gB] : 0ull);
          int c = 0;
          while (c < kMlSkip - 1 && (forb & (1ull << c)))
            ++c;
          mlPacked[idx] = (mlPacked[idx] & ~(63ll << shift)) | ((long long)c << shift);
          mask[gA] |= 1ull << c;
          if (gB >= 0)
            mask[gB] |= 1ull << c;
        }
        if (rem == prevRemaining)
          break;
        prevRemaining = rem;
        remaining = rem;
      }
      for (int idx = 0; idx < nm; ++idx) {
        const int c = (int)((mlPacked[idx] >> shift) & 63);
        if (c != kMlSkip && c > maxc)
          maxc = c;
      }
      H.push_back(MlLevel{groupOff, ngNew, parentOff, maxc + 1});
      parentOff += ngPrev;
      groupOff += ngNew;
      ngPrev = ngNew;
      if (ngNew <= 32)
        break;
    }
    return H;
  }
  void mlCoarseCycle(int nm, const std::vector<MlLevel>& H, R& maxQS, int coarseSweeps) {  // :331-478
    for (int i = 0; i < numReal; ++i)
      mlGrp[i] = i;
    for (int lvl = 1; lvl <= (int)H.size(); ++lvl) {
      const MlLevel& L = H[lvl - 1];
      const int off = L.groupOff, shift = 6 * (lvl - 1);
      for (int i = 0; i < numReal; ++i)
        mlGrp[i] = mlParent[L.parentOff + mlGrp[i]];
      for (int g = 0; g < L.numGroups; ++g)
        mlVelG[off + g] = V3<R>{0, 0, 0};
      for (int i = 0; i < numReal; ++i) {
        const R m = mlEffMass(invMass[i]);
        V3<R>& vg = mlVelG[off + mlGrp[i]];
        vg.x += m * velPred[i].x;
        vg.y += m * velPred[i].y;
        vg.z += m * velPred[i].z;
      }
      for (int g = 0; g < L.numGroups; ++g) {
        const R invM = R(1) / mlMassG[off + g];
        mlVelG[off + g].x *= invM;
        mlVelG[off + g].y *= invM;
        mlVelG[off + g].z *= invM;
        mlVelG0[off + g] = mlVelG[off + g];
      }
      for (int sw = 0; sw < coarseSweeps; ++sw)
        for (int color = 0; color < L.numColors; ++color)
          for (int idx = 0; idx < nm; ++idx) {
            if ((int)((mlPacked[idx] >> shift) & 63) != color)
              continue;
            const Manifold<R>& m = manifolds[idx];
            const int gA = mlGrp[realIdx[m.a]];
            const int gB = m.b >= 0 ? mlGrp[realIdx[m.b]] : -1;
            const R invN = R(1) / static_cast<R>(m.np);
            const V3<R> N = m.N;
            const R lenN = std::sqrt(dot(N, N));
            if (lenN < R(1e-9))
              continue;
            const V3<R> rAa = mul(m.rA, invN), rBa = mul(m.rB, invN);
            const V3<R> dc = gB < 0 ? rAa : sub(rAa, rBa);
            const V3<R> vA = mlVelG[off + gA];
            const V3<R> vB = gB >= 0 ? mlVelG[off + gB] : mul(m.wv, invN);
            const R vn = dot(sub(vA, vB), N);
            const R al = dot(N, dc);
            const R sgn = al > R(0) ? R(1) : R(-1);
            const R iA = mlInvMassG[off + gA];
            const R iB = gB >= 0 ? mlInvMassG[off + gB] : R(0);
            const R w = dot(N, N) * (iA + iB);
            if (w <= R(0))
              continue;
            const R dp = (sgn * vn) / w;
            const R pOld = lambdaAcc[idx];
            R pNew = pOld + dp;
            if (pNew < R(0))
              pNew = 0;
            const R d = pNew - pOld;
            if (d == R(0))
              continue;
            lambdaAcc[idx] = pNew;
            maxQS = std::max(maxQS, std::fabs(d) * w / lenN);
            const V3<R> J = mul(N, -sgn * d);
            V3<R>& a = mlVelG[off + gA];
            a.x += J.x * iA;
            a.y += J.y * iA;
            a.z += J.z * iA;
            if (gB >= 0) {
              V3<R>& b = mlVelG[off + gB];
              b.x -= J.x * iB;
              b.y -= J.y * iB;
              b.z -= J.z * iB;
            }
          }
      for (int i = 0; i < numReal; ++i) {
        const V3<R>& vg = mlVelG[off + mlGrp[i]];
        const V3<R>& v0 = mlVelG0[off + mlGrp[i]];
        velPred[i].x += vg.x - v0.x;
        velPred[i].y += vg.y - v0.y;
        velPred[i].z += vg.z - v0.z;
      }
    }
  }
  void multilevelStabilization(int nm, int ncol, V3<R> gHat, R vRestS, R gMag) {  // sim.hpp:303-356
    (void)gHat;
    const R qsThr = R(8) * dt * gMag;
    const std::vector<MlLevel> H = mlBuild(nm, qsThr);
    for (int it = 0; it < 2 * velIters; ++it) {
      R maxQS = 0;
      for (int c = 0; c < ncol; ++c)
        for (int i = 0; i < nm; ++i)
          if (mColor[i] == c)
            pgsOne(i, vRestS, maxApproach, &maxQS);
      if (!H.empty())
        mlCoarseCycle(nm, H, maxQS, 2);
      if (maxQS <= vRestS)
        break;
    }
  }

  void orderedStabilization(int nm, V3<R> gHat, R vRestS) {
    computeHeightLevels(nm, gHat);
    std::vector<int> key(nm), perm(nm);
    for (int i = 0; i < nm; ++i) {
      perm[i] = i;
      const Manifold<R>& m = manifolds[i];
      if (m.np <= 0 || mColor[i] < 0) {
        key[i] = INT_MAX;
        continue;
      }
      int h = heightLevel[realIdx[m.a]];
      if (m.b >= 0)
        h = std::min(h, heightLevel[realIdx[m.b]]);
      key[i] = std::min(h, 1023) * 64 + mColor[i];
    }
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return key[a] < key[b]; });
    std::vector<std::pair<int, int>> buckets;
    for (int b = 0; b < nm && key[perm[b]] != INT_MAX;) {
      int e = b + 1;
      while (e < nm && key[perm[e]] == key[perm[b]])
        ++e;
      buckets.emplace_back(b, e);
      b = e;
    }
    const int nb = (int)buckets.size();
    for (int it = 0; it < 2 * velIters; ++it) {
      maxApproach = 0;
      for (int pass = 0; pass < 2; ++pass)
        for (int q = 0; q < nb; ++q) {
          const auto [b, e] = buckets[pass == 0 ? q : nb - 1 - q];
          for (int t = b; t < e; ++t)
            pgsOne(perm[t], vRestS, maxApproach);
        }
      if (maxApproach <= vRestS)
        break;
    }
  }
  // output_sdf.hpp:25-196 (get_sdf_grid): over the domain box, every voxel starts at 100; each
  // particle writes min(analytic SDF x scale) over its band (bounding radius x scale x 1.2) and
  // marks the voxels nearer than that radius fixed; then max(res) x 4 Jacobi Eikonal sweeps
  // (spacing = the x voxel size) fill the rest, periodic axes wrapped. The particle scale alone
  // scales the shape (the global scale is not applied), and box shapes splat nothing, as in the
  // reference.
  std::vector<R> generateSdf(int rx, int ry, int rz) {
    const long total = (long)rx * ry * rz;
    const V3<R> origin = dmin;
    const V3<R> vox{(dmax.x - dmin.x) / R(rx), (dmax.y - dmin.y) / R(ry), (dmax.z - dmin.z) / R(rz)};
    std::vector<R> grid(total, R(100));
    std::vector<int> state(total, 0);
    for (int i = 0; i < numReal; ++i) {
      const V3<R> pw = pos[i];
      const V4<R> q = quat[i];
      const R sc = scale[i];
      const Shape<R>& shp = shapes[shapeId[i]];
      R rbound = R(1);
      if (shp.type == HCYL) {
        const R r = shp.par.x, h = shp.par.y;
        rbound = std::sqrt(r * r + (h * R(0.5)) * (h * R(0.5)));
      } else if (shp.type == SPHERE || shp.type == GRID) {
        rbound = shp.par.x;
      }
      rbound *= sc;
      rbound *= R(1.2);
      int mnx = (int)std::floor((pw.x - rbound - origin.x) / vox.x), mxx = (int)std::ceil((pw.x + rbound - origin.x) / vox.x);
      int mny = (int)std::floor((pw.y - rbound - origin.y) / vox.y), mxy = (int)std::ceil((pw.y + rbound - origin.y) / vox.y);
      int mnz = (int)std::floor((pw.z - rbound - origin.z) / vox.z), mxz = (int)std::ceil((pw.z + rbound - origin.z) / vox.z);
      if (!px)
        mnx = std::max(mnx, 0), mxx = std::min(mxx, rx - 1);
      if (!py)
        mny = std::max(mny, 0), mxy = std::min(mxy, ry - 1);
      if (!pz)
        mnz = std::max(mnz, 0), mxz = std::min(mxz, rz - 1);
      for (int z = mnz; z <= mxz; ++z)
        for (int y = mny; y <= mxy; ++y)
          for (int x = mnx; x <= mxx; ++x) {
            const V3<R> vp{origin.x + (R(x) + R(0.5)) * vox.x, origin.y + (R(y) + R(0.5)) * vox.y,
                           origin.z + (R(z) + R(0.5)) * vox.z};
            const V3<R> pl = mul(invrot(q, sub(vp, pw)), R(1) / sc);
            R distc = R(100);
            if (shp.type == HCYL)
              distc = sdfHollowCyl(pl, shp.par);
            else if (shp.type == SPHERE)
              distc = sdfSphere(pl, shp.par);
            else if (shp.type == GRID)
              distc = sdfShape(pl, shp, sdfGrid.data());
            const R dist = distc * sc;
            const int wx = (x % rx + rx) % rx, wy = (y % ry + ry) % ry, wz = (z % rz + rz) % rz;
            if ((!px && (x < 0 || x >= rx)) || (!py && (y < 0 || y >= ry)) || (!pz && (z < 0 || z >= rz)))
              continue;
            const long vi = (long)wz * rx * ry + (long)wy * rx + wx;
            grid[vi] = std::min(grid[vi], dist);
            if (dist < rbound)
              state[vi] = 1;
          }
    }
    std::vector<R> out(total);
    const int iters = std::max(std::max(rx, ry), rz) * 4;
    const R h = vox.x;
    for (int it = 0; it < iters; ++it) {
      for (long idx = 0; idx < total; ++idx)
        out[idx] = eikonalCell(grid, state, idx, rx, ry, rz, h);
      grid.swap(out);
    }
    return grid;
  }
  R eikonalCell(const std::vector<R>& in, const std::vector<int>& st, long idx, int rx, int ry, int rz, R h) const {
    if (st[idx] == 1)
      return in[idx];
    const long sy = rx, sz = (long)rx * ry;
    const int z = (int)(idx / sz);
    const long rem = idx % sz;
    const int y = (int)(rem / sy), x = (int)(rem % sy);
    R xm = 100, xp = 100, ym = 100, yp = 100, zm = 100, zp = 100;
    if (x > 0)
      xm = in[idx - 1];
    else if (px)
      xm = in[idx - 1 + rx];
    if (x < rx - 1)
      xp = in[idx + 1];
    else if (px)
      xp = in[idx + 1 - rx];
    if (y > 0)
      ym = in[idx - sy];
    else if (py)
      ym = in[(long)z * sz + (long)(ry - 1) * sy + x];
    if (y < ry - 1)
      yp = in[idx + sy];
    else if (py)
      yp = in[(long)z * sz + x];
    if (z > 0)
      zm = in[idx - sz];
    else if (pz)
      zm = in[(long)(rz - 1) * sz + (long)y * sy + x];
    if (z < rz - 1)
      zp = in[idx + sz];
    else if (pz)
      zp = in[(long)y * sy + x];
    R a = std::fmin(xm, xp), b = std::fmin(ym, yp), c = std::fmin(zm, zp);
    if (a > b)
      std::swap(a, b);
    if (b > c)
      std::swap(b, c);
    if (a > b)
      std::swap(a, b);
    R u = 100, u1 = a + h;
    if (u1 <= b) {
      u = u1;
    } else {
      const R d2 = R(2) * h * h - (a - b) * (a - b);
      const R u2 = (d2 < R(0)) ? R(100) : (a + b + std::sqrt(d2)) * R(0.5);
      if (u2 <= c) {
        u = u2;
      } else {
        const R s = a + b + c, qd = s * s - R(3) * (a * a + b * b + c * c - h * h);
        u = (qd < R(0)) ? R(100) : (s + std::sqrt(qd)) / R(3);
      }
    }
    return u;
  }
  void commitLedger(int nm) {  // :160-192
    if (nm <= 0)
      return;
    std::vector<int> perm(nm);
    std::iota(perm.begin(), perm.end(), 0);
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return pairKeys[a] < pairKeys[b]; });
    for (int i = 0; i < nm; ++i) {
      prevPairKeys[i] = pairKeys[perm[i]];
      prevLambda[i] = lambdaAcc[perm[i]];
      prevLambdaT[i] = lambdaT[perm[i]];
    }
  }
  void commitPosImpulse(int nc, int nm) {  // :501-538 (scratch = vn0, as the reference passes)
    for (int i = 0; i < nm; ++i)
      vn0[i] = 0;
    for (int i = 0; i < nc; ++i) {
      const R l = posLambdaContact[i];
      if (l != R(0))
        vn0[contactSlot[i]] += l / dt;
    }
    for (int i = 0; i < nm; ++i) {
      const u64 k = pairKeys[i];
      if (k == ~0ull)
        continue;
      const int lo = lowerBound(prevPairKeys, prevPairCount, k);
      if (lo < prevPairCount && prevPairKeys[lo] == k)
        prevPosImpulse[lo] = vn0[i];
    }
  }

  // ---------------- colouring (src/solver_velocity.hpp:277-374, solver_position.hpp:155-241) ----
  static long long colorKey(int idx) {  // contact_preprocessing.hpp:310-317
    unsigned z = (unsigned)idx + 0x9e3779b9u;
    z = (z ^ (z >> 16)) * 0x21f0aaadu;
    z = (z ^ (z >> 15)) * 0x735a2d97u;
    z ^= (z >> 15);
    return ((long long)(z & 0x7fffffffu) << 32) | (unsigned)idx;
  }
  // Generic Jones-Plassmann rounds over edges (ea, eb) (eb < 0: boundary); colour[] preset to -2
  // (inactive) or -1 (to colour). Returns max colour + 1 (max over all entries, as the reference's
  // Max reduction); `leftover` = entries still -1.
  template <class Ends>
  int jpColor(int ne, int nb, std::vector<int>& col, Ends ends, int& leftover) {
    for (int i = 0; i < nb; ++i)
      bodyMask[i] = 0;
    int remaining = 1, prevRem = -1;
    const int maxRounds = nb + 2;
    for (int round = 0; round < maxRounds && remaining > 0; ++round) {
      for (int i = 0; i < nb; ++i)
        bodyWinner[i] = -1;
      for (int i = 0; i < ne; ++i) {
        if (col[i] != -1)
          continue;
        int ea, eb;
        ends(i, ea, eb);
        const long long k = colorKey(i);
        if (k > bodyWinner[ea])
          bodyWinner[ea] = k;
        if (eb >= 0 && k > bodyWinner[eb])
          bodyWinner[eb] = k;
      }
      int rem = 0;
      for (int i = 0; i < ne; ++i) {
        if (col[i] != -1)
          continue;
        int ea, eb;
        ends(i, ea, eb);
        const long long k = colorKey(i);
        if (bodyWinner[ea] != k || (eb >= 0 && bodyWinner[eb] != k)) {
          ++rem;
          continue;
        }
        u64 forb = bodyMask[ea];
        if (eb >= 0)
          forb |= bodyMask[eb];
        int c = 0;
        while (c < 62 && (forb & (1ull << c)))
          ++c;
        col[i] = c;
        bodyMask[ea] |= 1ull << c;
        if (eb >= 0)
          bodyMask[eb] |= 1ull << c;
      }
      if (rem == prevRem)
        break;
      prevRem = rem;
      remaining = rem;
    }
    int mx = std::numeric_limits<int>::lowest();
    leftover = 0;
    for (int i = 0; i < ne; ++i) {
      mx = std::max(mx, col[i]);
      if (col[i] == -1)
        ++leftover;
    }
    return mx + 1;
  }
  int colorManifolds(int nm, int& leftover) {
    leftover = 0;
    if (nm <= 0 || numReal <= 0)
      return 0;
    for (int i = 0; i < nm; ++i) {
      const Manifold<R>& m = manifolds[i];
      if (m.np <= 0 || (m.b >= 0 && realIdx[m.a] > realIdx[m.b]))
        mColor[i] = -2;
      else
        mColor[i] = -1;
    }
    return jpColor(nm, numReal, mColor,
                   [&](int i, int& ea, int& eb) {
                     ea = realIdx[manifolds[i].a];
                     eb = manifolds[i].b >= 0 ? realIdx[manifolds[i].b] : -1;
                   },
                   leftover);
  }
  int colorContacts(int nc, int nb, int& leftover) {
    leftover = 0;
    if (nc <= 0 || nb <= 0)
      return 0;
    for (int i = 0; i < nc; ++i)
      cColor[i] = -1;
    return jpColor(nc, nb, cColor,
                   [&](int i, int& ea, int& eb) {
                     ea = contacts[i].a;
                     eb = contacts[i].b;
                   },
                   leftover);
  }

  // ---------------- velocity solve (src/solver_velocity.hpp) ----------------
  // solver_velocity.hpp:28-34
  static R genInvMass(V3<R> tau, V3<R> iI, V4<R> q) {
    if (iI.x == iI.y && iI.y == iI.z)
      return dot(tau, tau) * iI.x;
    const V3<R> t = invrot(q, tau);
    return t.x * t.x * iI.x + t.y * t.y * iI.y + t.z * t.z * iI.z;
  }
  // dw_world = R (invI_local * (R^T J))
  static V3<R> angDelta(V4<R> q, V3<R> J, V3<R> iI) {
    const V3<R> Jl = invrot(q, J);
    const V3<R> dwl{Jl.x * iI.x, Jl.y * iI.y, Jl.z * iI.z};
    return rot(q, dwl);
  }
  struct MView {  // per-manifold derived quantities shared by the velocity kernels
    int ra, rb;
    R imA, imB;
    V3<R> iIA, iIB;
    V4<R> qA, qB;
    R invN;
    V3<R> N, TA, TB, rAa, rBa, dc;
  };
  MView view(const Manifold<R>& m) const {
    MView v;
    v.ra = realIdx[m.a];
    v.rb = m.b >= 0 ? realIdx[m.b] : m.b;
    v.imA = invMass[v.ra];
    v.imB = m.b >= 0 ? invMass[v.rb] : R(0);
    v.iIA = invI[v.ra];
    v.iIB = m.b >= 0 ? invI[v.rb] : V3<R>{0, 0, 0};
    v.qA = quat[v.ra];
    v.qB = m.b >= 0 ? quat[v.rb] : V4<R>{0, 0, 0, 1};
    v.invN = R(1) / static_cast<R>(m.np);
    v.N = m.N;
    v.TA = m.TA;
    v.TB = m.TB;
    v.rAa = mul(m.rA, v.invN);
    v.rBa = mul(m.rB, v.invN);
    v.dc = (m.b < 0) ? v.rAa : sub(v.rAa, v.rBa);
    return v;
  }
  // :38-226 Jacobi (colorFilter: only manifolds whose colour == filter, when filt)
  void solveVelocityJacobi(int nm, R vRest, bool filt, int filter) {
    for (int idx = 0; idx < nm; ++idx) {
      if (filt && mColor[idx] != filter)
        continue;
      const Manifold<R>& m = manifolds[idx];
      if (m.np <= 0)
        continue;
      const int ra = realIdx[m.a];
      int rb = m.b;
      if (m.b >= 0) {
        rb = realIdx[m.b];
        if (ra > rb)
          continue;
      }
      const MView v = view(m);
      V3<R> vA = velPred[ra], wA = angVelPred[ra], vB{0, 0, 0}, wB{0, 0, 0};
      if (m.b >= 0) {
        vB = velPred[rb];
        wB = angVelPred[rb];
      }
      R e = eN;
      if (m.b < 0)
        vB = mul(m.wv, v.invN);
      {
        const R ra2 = m.e * v.invN;
        if (ra2 >= R(0))
          e = ra2;
      }
      const R lenN = std::sqrt(dot(v.N, v.N));
      if (lenN < R(1e-9))
        continue;
      const V3<R> vG = mul(v.dc, growthRate);
      R vn = dot(vA, v.N) + dot(wA, v.TA) + dot(vB, neg(v.N)) + dot(wB, v.TB);
      vn += dot(vG, v.N);
      const R al = dot(v.N, v.dc);
      if (al > R(0)) {
        if (vn < R(0))
          continue;
      } else {
        if (vn > R(0))
          continue;
      }
      const R Nsq = dot(v.N, v.N);
      const R wAn = Nsq * v.imA + genInvMass(v.TA, v.iIA, v.qA);
      const R wBn = Nsq * v.imB + genInvMass(v.TB, v.iIB, v.qB);
      const R wT = wAn + wBn;
      if (wT <= R(0))
        continue;
      if (std::fabs(vn) < vRest * lenN)
        e = 0;
      const R lam = (-e * vn - vn) / wT;
      const V3<R> J = mul(v.N, lam), JA = mul(v.TA, lam), JB = mul(v.TB, lam);
      deltaVel[ra] = add(deltaVel[ra], mul(J, v.imA));
      deltaAngVel[ra] = add(deltaAngVel[ra], angDelta(v.qA, JA, v.iIA));
      if (m.b >= 0) {
        deltaVel[rb] = add(deltaVel[rb], mul(neg(J), v.imB));
        deltaAngVel[rb] = add(deltaAngVel[rb], angDelta(v.qB, JB, v.iIB));
        constraintCounts[rb] += 1;
      }
      constraintCounts[ra] += 1;
    }
  }
  // :234-255
  void applyVelocityDeltasAveraged(int n) {
    for (int i = 0; i < n; ++i) {
      const int c = constraintCounts[i];
      if (c <= 0)
        continue;
      const R f = std::fmin(R(1), R(2) / static_cast<R>(c));
      velPred[i] = add(velPred[i], mul(deltaVel[i], f));
      angVelPred[i] = add(angVelPred[i], mul(deltaAngVel[i], f));
      deltaVel[i] = deltaAngVel[i] = V3<R>{0, 0, 0};
      constraintCounts[i] = 0;
    }
  }
  // :390-447
  void computeVn0(int nm) {
    for (int idx = 0; idx < nm; ++idx) {
      const Manifold<R>& m = manifolds[idx];
      if (m.np <= 0)
        continue;
      const int ra = realIdx[m.a];
      if (m.b >= 0 && ra > realIdx[m.b])
        continue;
      const MView v = view(m);
      const V3<R> vA = velPred[ra], wA = angVelPred[ra];
      V3<R> vB{0, 0, 0}, wB{0, 0, 0};
      if (m.b >= 0) {
        vB = velPred[realIdx[m.b]];
        wB = angVelPred[realIdx[m.b]];
      } else {
        vB = mul(m.wv, v.invN);
      }
      const V3<R> vG = mul(v.dc, growthRate);
      R vn = dot(vA, v.N) + dot(wA, v.TA) + dot(vB, neg(v.N)) + dot(wB, v.TB);
      vn += dot(vG, v.N);
      vn0[idx] = vn;
      const R lenN = std::sqrt(dot(v.N, v.N));
      V3<R> vt{0, 0, 0};
      if (lenN > R(1e-9)) {
        const V3<R> nh = mul(v.N, R(1) / lenN);
        const int rb2 = m.b >= 0 ? realIdx[m.b] : -1;
        const V3<R> wAv = angVelPred[ra];
        const V3<R> wBv = rb2 >= 0 ? angVelPred[rb2] : V3<R>{0, 0, 0};
        const V3<R> vr = sub(add(vA, cross(wAv, v.rAa)), add(vB, cross(wBv, v.rBa)));
        vt = sub(vr, mul(nh, dot(vr, nh)));
      }
      vt0[idx] = vt;
    }
  }
  // :456-495
  void computeSideFlags(int nm, V3<R> gHat, R riseThr, R approachThr) {
    for (int idx = 0; idx < nm; ++idx) {
      const unsigned char was = persistent[idx];
      sideFlags[idx] = 0;
      const Manifold<R>& m = manifolds[idx];
      if (m.np <= 0 || m.b < 0 || was == 0)
        continue;
      if (std::fabs(vn0[idx]) > approachThr)
        continue;
      const int ra = realIdx[m.a], rb = realIdx[m.b];
      if (ra > rb)
        continue;
      const V3<R> dx = sub(posPred[m.a], posPred[m.b]);
      const R up = -(dx.x * gHat.x + dx.y * gHat.y + dx.z * gHat.z);
      const R thr = R(0.3) * std::sqrt(dot(dx, dx));
      if (up > thr && -dot(velPred[rb], gHat) <= riseThr && grounded[rb] > 0)
        sideFlags[idx] = 1;
      else if (up < -thr && -dot(velPred[ra], gHat) <= riseThr && grounded[ra] > 0)
        sideFlags[idx] = 2;
    }
  }
  // :498-605
  void warmStartApply(int nm) {
    for (int idx = 0; idx < nm; ++idx) {
      const R p = lambdaAcc[idx];
      V3<R> lt = lambdaT[idx];
      const bool hasT = lt.x != R(0) || lt.y != R(0) || lt.z != R(0);
      if (p == R(0) && !hasT)
        continue;
      const Manifold<R>& m = manifolds[idx];
      if (m.np <= 0)
        continue;
      const int ra = realIdx[m.a];
      const int rb = m.b >= 0 ? realIdx[m.b] : m.b;
      if (m.b >= 0 && ra > rb)
        continue;
      const R invN = R(1) / static_cast<R>(m.np);
      const V3<R> rAa = mul(m.rA, invN), rBa = mul(m.rB, invN);
      const V3<R> dc = (m.b < 0) ? rAa : sub(rAa, rBa);
      const R al = dot(m.N, dc);
      const R sgn = (al > R(0)) ? R(1) : R(-1);
      const R lam = -sgn * p;
      const V3<R> J = mul(m.N, lam);
      const R imA = invMass[ra];
      const R imB = m.b >= 0 ? invMass[rb] : R(0);
      velPred[ra] = add(velPred[ra], mul(J, imA));
      angVelPred[ra] = add(angVelPred[ra], angDelta(quat[ra], mul(m.TA, lam), invI[ra]));
      if (m.b >= 0) {
        velPred[rb] = add(velPred[rb], mul(neg(J), imB));
        angVelPred[rb] = add(angVelPred[rb], angDelta(quat[rb], mul(m.TB, lam), invI[rb]));
      }
      if (hasT) {
        const R l2 = std::sqrt(dot(m.N, m.N));
        if (l2 > R(1e-9)) {
          const V3<R> nh = mul(m.N, R(1) / l2);
          lt = sub(lt, mul(nh, dot(lt, nh)));
        }
        lambdaT[idx] = lt;
        velPred[ra] = add(velPred[ra], mul(lt, imA));
        angVelPred[ra] = add(angVelPred[ra], angDelta(quat[ra], cross(rAa, lt), invI[ra]));
        if (m.b >= 0) {
          velPred[rb] = add(velPred[rb], mul(neg(lt), imB));
          angVelPred[rb] = add(angVelPred[rb], angDelta(quat[rb], cross(rBa, mul(lt, R(-1))), invI[rb]));
        }
      }
    }
  }
  // :641-858 PGSManifoldSweep::solveOne
  // maxQS (the multilevel pass): also the largest correction on quasi-static contacts,
  // |vn0| <= 4 vRest |N| (src/solver_velocity.hpp:722-723, 829-830)
  void pgsOne(int idx, R vRest, R& maxApp, R* maxQS = nullptr) {
    const Manifold<R>& m = manifolds[idx];
    const MView v = view(m);
    const int ra = v.ra, rb = v.rb;
    const V3<R> vA = velPred[ra], wA = angVelPred[ra];
    V3<R> vB{0, 0, 0}, wB{0, 0, 0};
    R e = eN;
    if (m.b >= 0) {
      vB = velPred[rb];
      wB = angVelPred[rb];
    } else {
      vB = mul(m.wv, v.invN);
    }
    {
      const R ra2 = m.e * v.invN;
      if (ra2 >= R(0))
        e = ra2;
    }
    const R lenN = std::sqrt(dot(v.N, v.N));
    if (lenN < R(1e-9))
      return;
    const V3<R> vG = mul(v.dc, growthRate);
    R vn = dot(vA, v.N) + dot(wA, v.TA) + dot(vB, neg(v.N)) + dot(wB, v.TB);
    vn += dot(vG, v.N);
    const R al = dot(v.N, v.dc);
    const R sgn = (al > R(0)) ? R(1) : R(-1);
    const R Nsq = dot(v.N, v.N);
    R wAn = Nsq * v.imA + genInvMass(v.TA, v.iIA, v.qA);
    R wBn = Nsq * v.imB + genInvMass(v.TB, v.iIB, v.qB);
    bool applyA = true, applyB = true;
    const unsigned char sf = sideFlags[idx];
    if (sf == 1) {
      wBn = 0;
      applyB = false;
      e = 0;
    } else if (sf == 2) {
      wAn = 0;
      applyA = false;
      e = 0;
    }
    const R wT = wAn + wBn;
    if (wT <= R(0))
      return;
    const R v0 = sgn * vn0[idx];
    if (std::fabs(vn0[idx]) < vRest * lenN)
      e = 0;
    const R target = (v0 > R(0)) ? -e * v0 : R(0);
    const R vt = sgn * vn;
    const R dp = (vt - target) / wT;
    const R pOld = lambdaAcc[idx];
    R pNew = pOld + dp;
    if (pNew < R(0))
      pNew = 0;
    const R dA = pNew - pOld;
    if (dA != R(0)) {
      lambdaAcc[idx] = pNew;
      maxApp = std::max(maxApp, std::fabs(dA) * wT / lenN);
      if (maxQS && std::fabs(vn0[idx]) <= R(4) * vRest * lenN)
        *maxQS = std::max(*maxQS, std::fabs(dA) * wT / lenN);
      const R lam = -sgn * dA;
      const V3<R> J = mul(v.N, lam), JA = mul(v.TA, lam), JB = mul(v.TB, lam);
      if (applyA) {
        velPred[ra] = add(velPred[ra], mul(J, v.imA));
        angVelPred[ra] = add(angVelPred[ra], angDelta(v.qA, JA, v.iIA));
      }
      if (m.b >= 0 && applyB) {
        velPred[rb] = add(velPred[rb], mul(neg(J), v.imB));
        angVelPred[rb] = add(angVelPred[rb], angDelta(v.qB, JB, v.iIB));
      }
    }
    // friction cone
    R muE = mu;
    const R fa = m.mu * v.invN;
    if (fa >= R(0))
      muE = fa;
    const V3<R> ltOld = lambdaT[idx];
    const bool haveOld = ltOld.x != R(0) || ltOld.y != R(0) || ltOld.z != R(0);
    if (!(muE > R(0) || haveOld))
      return;
    const V3<R> nh = mul(v.N, R(1) / lenN);
    const V3<R> vA2 = velPred[ra], wA2 = angVelPred[ra];
    V3<R> vB2{0, 0, 0}, wB2{0, 0, 0};
    if (m.b >= 0) {
      vB2 = velPred[rb];
      wB2 = angVelPred[rb];
    } else {
      vB2 = mul(m.wv, v.invN);
    }
    const V3<R> vr = sub(add(vA2, cross(wA2, v.rAa)), add(vB2, cross(wB2, v.rBa)));
    const V3<R> vtv = sub(vr, mul(nh, dot(vr, nh)));
    R beta = eT;
    if (beta != R(0) && (sf != 0 || std::fabs(vn0[idx]) < vRest * lenN))
      beta = 0;
    V3<R> err = vtv;
    if (beta != R(0)) {
      V3<R> w0 = vt0[idx];
      w0 = sub(w0, mul(nh, dot(w0, nh)));
      err = add(vtv, mul(w0, beta));
    }
    const R vl = std::sqrt(dot(err, err));
    V3<R> ltNew = ltOld;
    R wTt = v.imA + v.imB;
    if (vl > R(1e-9)) {
      const V3<R> th = mul(err, R(1) / vl);
      const R wAt = (sf == 2) ? R(0) : v.imA + genInvMass(cross(v.rAa, th), v.iIA, v.qA);
      const R wBt = (sf == 1 || m.b < 0) ? R(0) : v.imB + genInvMass(cross(v.rBa, th), v.iIB, v.qB);
      wTt = wAt + wBt;
      if (wTt > R(1e-9))
        ltNew = add(ltOld, mul(th, -vl / wTt));
    }
    ltNew = sub(ltNew, mul(nh, dot(ltNew, nh)));
    R nTot = std::fmax(lambdaAcc[idx], R(0)) * lenN;
    if (std::fabs(vn0[idx]) < vRest * lenN)
      nTot += std::fmax(posImpulse[idx], R(0));
    const R bound = muE * nTot;
    const R ll = std::sqrt(dot(ltNew, ltNew));
    if (ll > bound)
      ltNew = (bound > R(0)) ? mul(ltNew, bound / ll) : V3<R>{0, 0, 0};
    const V3<R> d = sub(ltNew, ltOld);
    if (d.x != R(0) || d.y != R(0) || d.z != R(0)) {
      lambdaT[idx] = ltNew;
      const R dl = std::sqrt(dot(d, d));
      if (wTt > R(1e-9)) {
        maxApp = std::max(maxApp, dl * wTt);
        if (maxQS && std::fabs(vn0[idx]) <= R(4) * vRest * lenN)
          *maxQS = std::max(*maxQS, dl * wTt);
      }
      if (applyA) {
        velPred[ra] = add(velPred[ra], mul(d, v.imA));
        angVelPred[ra] = add(angVelPred[ra], angDelta(v.qA, cross(v.rAa, d), v.iIA));
      }
      if (m.b >= 0 && applyB) {
        velPred[rb] = add(velPred[rb], mul(neg(d), v.imB));
        angVelPred[rb] = add(angVelPred[rb], angDelta(v.qB, cross(v.rBa, mul(d, R(-1))), v.iIB));
      }
    }
  }
  void solveVelocityPGS(int nm, int ncol, R vRest) {  // :861-904
    for (int c = 0; c < ncol; ++c)
      for (int i = 0; i < nm; ++i)
        if (mColor[i] == c)
          pgsOne(i, vRest, maxApproach);
  }
  // :989-1137 one-shot coloured GS (g = 0 path)
  void solveVelocityColoredGS(int nm, int ncol, R vRest) {
    for (int c = 0; c < ncol; ++c)
      for (int idx = 0; idx < nm; ++idx) {
        if (mColor[idx] != c)
          continue;
        const Manifold<R>& m = manifolds[idx];
        const MView v = view(m);
        const int ra = v.ra, rb = v.rb;
        const V3<R> vA = velPred[ra], wA = angVelPred[ra];
        V3<R> vB{0, 0, 0}, wB{0, 0, 0};
        if (m.b >= 0) {
          vB = velPred[rb];
          wB = angVelPred[rb];
        }
        R e = eN;
        if (m.b < 0)
          vB = mul(m.wv, v.invN);
        {
          const R ra2 = m.e * v.invN;
          if (ra2 >= R(0))
            e = ra2;
        }
        const R lenN = std::sqrt(dot(v.N, v.N));
        if (lenN < R(1e-9))
          continue;
        const V3<R> vG = mul(v.dc, growthRate);
        R vn = dot(vA, v.N) + dot(wA, v.TA) + dot(vB, neg(v.N)) + dot(wB, v.TB);
        vn += dot(vG, v.N);
        const R al = dot(v.N, v.dc);
        if (al > R(0)) {
          if (vn < R(0))
            continue;
        } else {
          if (vn > R(0))
            continue;
        }
        const R Nsq = dot(v.N, v.N);
        const R wAn = Nsq * v.imA + genInvMass(v.TA, v.iIA, v.qA);
        const R wBn = Nsq * v.imB + genInvMass(v.TB, v.iIB, v.qB);
        const R wT = wAn + wBn;
        if (wT <= R(0))
          continue;
        maxApproach = std::max(maxApproach, std::fabs(vn) / lenN);
        if (std::fabs(vn) < vRest * lenN)
          e = 0;
        const R lam = (-e * vn - vn) / wT;
        const V3<R> J = mul(v.N, lam), JA = mul(v.TA, lam), JB = mul(v.TB, lam);
        velPred[ra] = add(velPred[ra], mul(J, v.imA));
        angVelPred[ra] = add(angVelPred[ra], angDelta(v.qA, JA, v.iIA));
        if (m.b >= 0) {
          velPred[rb] = add(velPred[rb], mul(neg(J), v.imB));
          angVelPred[rb] = add(angVelPred[rb], angDelta(v.qB, JB, v.iIB));
        }
      }
  }

  // ---------------- legacy friction (src/solver_friction.hpp) ----------------
  static R computeW(V3<R> r, V3<R> d, R im, V3<R> iI) {  // solver_position.hpp:21-24
    const V3<R> rn = cross(r, d);
    return im + rn.x * rn.x * iI.x + rn.y * rn.y * iI.y + rn.z * rn.z * iI.z;
  }
  void accumulateNormalImpulse(int nc) {  // solver_friction.hpp:32-83
    for (int idx = 0; idx < nc; ++idx) {
      Contact<R>& c = contacts[idx];
      if (c.b < 0) {
        const int A = c.a;
        const R im = invMass[A];
        if (im <= R(0))
          continue;
        const V3<R> iI = invI[A];
        const V3<R> vAc = add(velPred[A], cross(angVelPred[A], c.rA));
        const R ap = -dot(sub(vAc, c.bvel), c.n);
        if (ap <= R(0))
          continue;
        const R wn = computeW(c.rA, c.n, im, iI);
        if (wn > R(1e-6))
          c.lamN += ap / wn;
        continue;
      }
      const int ra = realIdx[c.a], rb = realIdx[c.b];
      if (ra > rb)
        continue;
      const R imA = invMass[ra], imB = invMass[rb];
      const V3<R> iA = invI[ra], iB = invI[rb];
      const V3<R> vAc = add(velPred[ra], cross(angVelPred[ra], c.rA));
      const V3<R> vBc = add(velPred[rb], cross(angVelPred[rb], c.rB));
      const V3<R> vr = add(sub(vAc, vBc), mul(sub(c.rA, c.rB), growthRate));
      const R ap = -dot(vr, c.n);
      if (ap <= R(0))
        continue;
      const R wn = computeW(c.rA, c.n, imA, iA) + computeW(c.rB, c.n, imB, iB);
      if (wn > R(1e-6))
        c.lamN += ap / wn;
    }
  }
  void computePlaneLoad(int nc) {  // solver_friction.hpp:87-120
    std::fill(planeFric.begin(), planeFric.end(), R(0));
    for (int idx = 0; idx < nc; ++idx) {
      Contact<R>& c = contacts[idx];
      if (c.b >= 0)
        continue;
      const int A = c.a;
      const R im = invMass[A];
      if (im <= R(0))
        continue;
      const V3<R> vAc = add(velPred[A], cross(angVelPred[A], c.rA));
      const R ap = -dot(sub(vAc, c.bvel), c.n);
      if (ap <= R(0))
        continue;
      const R wn = computeW(c.rA, c.n, im, invI[A]);
      c.lamN = (wn > R(1e-6)) ? ap / wn : R(0);
      planeFric[2 * A] = std::max(planeFric[2 * A], ap / im);
    }
  }
  void countFrictionContacts(int nc) {  // solver_friction.hpp:123-138
    for (int idx = 0; idx < nc; ++idx) {
      const Contact<R>& c = contacts[idx];
      if (c.lamN <= R(0))
        continue;
      planeFric[2 * realIdx[c.a] + 1] += R(1);
      if (c.b >= 0)
        planeFric[2 * realIdx[c.b] + 1] += R(1);
    }
  }
  void solveContactFriction(int nc) {  // solver_friction.hpp:142-220
    std::fill(deltaVel.begin(), deltaVel.end(), V3<R>{0, 0, 0});
    std::fill(deltaAngVel.begin(), deltaAngVel.end(), V3<R>{0, 0, 0});
    for (int idx = 0; idx < nc; ++idx) {
      const Contact<R>& c = contacts[idx];
      const R ln = c.lamN;
      if (ln <= R(0))
        continue;
      const int ra = realIdx[c.a];
      const int rb = c.b >= 0 ? realIdx[c.b] : -1;
      const R imA = invMass[ra], imB = c.b >= 0 ? invMass[rb] : R(0);
      const V3<R> iA = invI[ra], iB = c.b >= 0 ? invI[rb] : V3<R>{0, 0, 0};
      const V3<R> vAc = add(velPred[ra], cross(angVelPred[ra], c.rA));
      V3<R> vBc{0, 0, 0};
      if (c.b >= 0)
        vBc = add(velPred[rb], cross(angVelPred[rb], c.rB));
      else
        vBc = c.bvel;
      const V3<R> vr = sub(vAc, vBc);
      const R vn = dot(vr, c.n);
      const V3<R> vt = sub(vr, mul(c.n, vn));
      const R vl = std::sqrt(dot(vt, vt));
      if (vl < R(1e-7))
        continue;
      const V3<R> t = mul(vt, R(1) / vl);
      const V3<R> rnA = cross(c.rA, t), rnB = cross(c.rB, t);
      const R wt = imA + imB + rnA.x * rnA.x * iA.x + rnA.y * rnA.y * iA.y + rnA.z * rnA.z * iA.z +
                   rnB.x * rnB.x * iB.x + rnB.y * rnB.y * iB.y + rnB.z * rnB.z * iB.z;
      if (wt < R(1e-6))
        continue;
      const R bound = ln;
      const R nA = planeFric[2 * ra + 1];
      const R nB = c.b >= 0 ? planeFric[2 * rb + 1] : R(0);
      const R invn = R(1) / std::fmax(std::fmax(nA, nB), R(1));
      R lt = -vl / wt;
      const R muE = (c.mu >= R(0)) ? c.mu : mu;
      const R maxf = muE * bound;
      if (lt < -maxf)
        lt = -maxf;
      lt *= invn;
      deltaVel[ra] = add(deltaVel[ra], V3<R>{t.x * lt * imA, t.y * lt * imA, t.z * lt * imA});
      deltaAngVel[ra] = add(deltaAngVel[ra], V3<R>{rnA.x * iA.x * lt, rnA.y * iA.y * lt, rnA.z * iA.z * lt});
      if (c.b >= 0) {
        deltaVel[rb] = add(deltaVel[rb], V3<R>{-t.x * lt * imB, -t.y * lt * imB, -t.z * lt * imB});
        deltaAngVel[rb] = add(deltaAngVel[rb], V3<R>{-rnB.x * iB.x * lt, -rnB.y * iB.y * lt, -rnB.z * iB.z * lt});
      }
    }
  }

  // ---------------- position solve (src/solver_position.hpp) ----------------
  // Shared per-contact constraint evaluation (:55-99 / :266-307). Returns false when inactive.
  bool posConstraint(const Contact<R>& c, V3<R>& n, R& C, R& wT) const {
    const int A = c.a, B = c.b;
    const R imA = invMass[A], imB = B >= 0 ? invMass[B] : R(0);
    const V3<R> pA = posPred[A];
    const V4<R> qA = quatPred[A];
    V3<R> pB{0, 0, 0};
    V4<R> qB{0, 0, 0, 1};
    if (B >= 0) {
      pB = posPred[B];
      qB = quatPred[B];
    }
    const V4<R> qAd = qmul(qA, qinv(quat[A]));
    const V3<R> rA = rot(qAd, c.rA);
    V3<R> rB = c.rB;
    n = c.n;
    if (B >= 0) {
      const V4<R> qBd = qmul(qB, qinv(quat[B]));
      rB = rot(qBd, rB);
      n = rot(qBd, n);
    }
    if (B < 0) {
      n = c.n;
      C = dot(sub(add(pA, rA), c.rB), n);
    } else {
      C = dot(sub(add(pA, rA), add(pB, rB)), n);
    }
    if (C >= R(0))
      return false;
    const V3<R> iA = invI[A], iB = B >= 0 ? invI[B] : V3<R>{0, 0, 0};
    wT = computeW(rA, n, imA, iA) + computeW(rB, n, imB, iB);
    return true;
  }
  void solvePositionJacobi(int nc, bool filt, int filter) {  // :34-134
    for (int idx = 0; idx < nc; ++idx) {
      if (filt && cColor[idx] != filter)
        continue;
      const Contact<R>& c = contacts[idx];
      V3<R> n;
      R C = 0, wT = 0;
      if (!posConstraint(c, n, C, wT))
        continue;
      if (wT < R(1e-6))
        continue;
      const R dl = -C / wT;
      const R imA = invMass[c.a];
      deltaPos[c.a] = add(deltaPos[c.a], V3<R>{n.x * dl * imA, n.y * dl * imA, n.z * dl * imA});
      if (c.b >= 0) {
        const R imB = invMass[c.b];
        deltaPos[c.b] = add(deltaPos[c.b], V3<R>{-n.x * dl * imB, -n.y * dl * imB, -n.z * dl * imB});
        constraintCounts[c.b] += 1;
      }
      constraintCounts[c.a] += 1;
      if (C < R(0))
        maxOverlap = std::max(maxOverlap, -C);
    }
  }
  void solvePositionGS(int nc, int ncol) {  // :248-331
    for (int col = 0; col < ncol; ++col)
      for (int idx = 0; idx < nc; ++idx) {
        if (cColor[idx] != col)
          continue;
        const Contact<R>& c = contacts[idx];
        V3<R> n;
        R C = 0, wT = 0;
        if (!posConstraint(c, n, C, wT))
          continue;
        if (wT < R(1e-6))
          continue;
        const R dl = -C / wT;
        posLambdaContact[idx] += dl;
        const R imA = invMass[c.a];
        posPred[c.a] = add(posPred[c.a], V3<R>{n.x * dl * imA, n.y * dl * imA, n.z * dl * imA});
        if (c.b >= 0) {
          const R imB = invMass[c.b];
          posPred[c.b] = add(posPred[c.b], V3<R>{-n.x * dl * imB, -n.y * dl * imB, -n.z * dl * imB});
        }
        maxOverlap = std::max(maxOverlap, -C);
      }
  }

  // ---------------- the substep (src/sim.hpp:97-488) ----------------
  R maxOwnedRadius() const {  // sim.hpp:61-70
    if (numReal <= 0)
      return globalScale * baseRadius;
    R mx = std::numeric_limits<R>::lowest();
    for (int i = 0; i < numReal; ++i)
      mx = scale[i] > mx ? scale[i] : mx;
    return mx * globalScale * baseRadius;
  }
  void fillRadii() {
    for (int i = 0; i < numParticles; ++i)
      rad[i] = scale[i] * globalScale * baseRadius;
  }
  void resetGhosts(R band) {
    for (int i = 0; i < numReal; ++i)
      realIdx[i] = i;
    topGhost = numReal;
    ensureCapacity(ghostCapacity(numReal, band));
    generateGhosts(band);
    numParticles = topGhost;
  }
  void detectAll(R margin) {
    const int np = findCollisionsGrow(margin);
    contactCount = 0;
    maxOverlap = 0;
    detectContacts(np, margin);
    detectBoundary(margin);
    if (!walls.empty())
      detectWallSdf(margin);
  }

  void demStep() {
    if (growthFactor != R(-1) && growthRate != R(0)) {
      growthFactor *= std::exp(growthRate * dt);
      if (growthFactor > R(1))
        growthFactor = 1;
    }
    if (growthFactor > R(0))
      updateGrowthScales(numReal, growthFactor);
    const R maxRad = maxOwnedRadius();
    const R margin = R(0.1) * maxRad;
    predictVelocity(numReal);
    resetGhosts(maxRad);
    fillRadii();
    detectAll(margin);
    const int nc = contactCount;
    const int nm = reduceToManifolds(nc);

    const bool friction = (mu > R(0) || wallFrictionMax > R(0));
    const bool gNZ = (gravity.x != R(0) || gravity.y != R(0) || gravity.z != R(0));
    const bool legacyFriction = friction && !(gNZ && useGS);
    if (legacyFriction)
      computePlaneLoad(nc);
    int velLeft = 0;
    const int ncolV = useGS ? colorManifolds(nm, velLeft) : 0;
    const bool usePGS = gNZ && useGS;
    const R gMag = std::sqrt(gravity.x * gravity.x + gravity.y * gravity.y + gravity.z * gravity.z);
    const V3<R> gHat = gNZ ? V3<R>{gravity.x / gMag, gravity.y / gMag, gravity.z / gMag} : V3<R>{0, 0, 0};
    if (usePGS) {
      gatherWarm(nm);
      markPersistent(nm);
      updateGrounded(nm, gHat, 8, 8);
      for (int i = 0; i < nm; ++i)
        sideFlags[i] = 0;
      computeVn0(nm);
      warmStartApply(nm);
    }
    for (int it = 0; it < velIters; ++it) {
      if (legacyFriction)
        accumulateNormalImpulse(nc);
      const R vRest = R(2) * dt * std::sqrt(gravity.x * gravity.x + gravity.y * gravity.y + gravity.z * gravity.z);
      if (useGS) {
        maxApproach = 0;
        if (usePGS)
          solveVelocityPGS(nm, ncolV, vRest);
        else
          solveVelocityColoredGS(nm, ncolV, vRest);
        if (velLeft > 0) {
          solveVelocityJacobi(nm, vRest, true, -1);
          applyVelocityDeltasAveraged(numParticles);
        }
        if (maxApproach <= (usePGS ? R(0.02) * vRest : vRest))
          break;
      } else {
        solveVelocityJacobi(nm, vRest, false, 0);
        applyVelocityDeltasAveraged(numParticles);
      }
    }
    if (usePGS) {
      const R vRestS = R(2) * dt * gMag;
      if (stabMode != 0 && maxApproach > vRestS) {
        if (stabMode == 1) {
          computeSideFlags(nm, gHat, R(8) * dt * gMag, R(8) * dt * gMag);
          for (int it = 0; it < 2 * velIters; ++it) {
            maxApproach = 0;
            solveVelocityPGS(nm, ncolV, vRestS);
            if (maxApproach <= vRestS)
              break;
          }
        } else if (stabMode == 3) {
          for (int it = 0; it < 256; ++it) {
            maxApproach = 0;
            solveVelocityPGS(nm, ncolV, vRestS);
            if (maxApproach <= vRestS)
              break;
          }
        } else if (stabMode == 4) {
          orderedStabilization(nm, gHat, vRestS);
        } else {
          multilevelStabilization(nm, ncolV, gHat, vRestS, gMag);
        }
      }
    }
    if (usePGS) {
      commitLedger(nm);
      prevPairCount = nm;
    }
    if (legacyFriction) {
      countFrictionContacts(nc);
      solveContactFriction(nc);
      applyVelocityDeltas(numParticles);
    }
    applyVelocityAndPredictPosition(numParticles);
    int posLeft = 0;
    const int ncolP = useGS ? colorContacts(nc, numParticles, posLeft) : 0;
    const R posTol = R(1e-4) * baseRadius * globalScale;
    for (int i = 0; i < nc; ++i)
      posLambdaContact[i] = 0;
    for (int it = 0; it < posIters; ++it) {
      if (useGS) {
        maxOverlap = 0;
        solvePositionGS(nc, ncolP);
        if (posLeft > 0) {
          solvePositionJacobi(nc, true, -1);
          applyUpdates(numParticles);
        }
        if (maxOverlap < posTol)
          break;
      } else {
        solvePositionJacobi(nc, false, 0);
        applyUpdates(numParticles);
      }
    }
    if (usePGS && nm > 0)
      commitPosImpulse(nc, nm);
    finalCommit(numReal);
    if (thermoTau > R(0) && dt > R(0))
      thermostat(numReal);
  }

  // sim.hpp:494-541
  R computeOverlaps() {
    const R maxRad = maxOwnedRadius();
    const R margin = R(0.1) * maxRad;
    numParticles = numReal;
    posPred = pos;
    quatPred = quat;
    resetGhosts(maxRad);
    fillRadii();
    detectAll(margin);
    numParticles = numReal;
    return maxOverlap;
  }

  // ---------------- Hertz-Mindlin engine (src/solver_hertz.hpp, src/sim.hpp:545-750) ----------
  static R betaD(R e) {  // solver_hertz.hpp:41-48
    if (e <= R(0))
      return R(-1);
    if (e >= R(1))
      return R(0);
    const R le = std::log(e);
    return le / std::sqrt(le * le + R(9.8696044));
  }
  // solver_hertz.hpp:53-84
  static V3<R> hertzForce(R delta, V3<R> nh, V3<R> vr, R rS, R mS, R eS, R gS, R e, R muE, R dtt,
                          V3<R>& xi) {
    const R sq = std::sqrt(rS * delta);
    const R sn = R(2) * eS * sq;
    const R st = R(8) * gS * sq;
    const R kn = (R(4) / R(3)) * eS * sq;
    const R bd = betaD(e);
    const R etaN = R(-2) * R(0.9128709) * bd * std::sqrt(sn * mS);
    const R etaT = R(-2) * R(0.9128709) * bd * std::sqrt(st * mS);
    const R vn = dot(vr, nh);
    const R fs = kn * delta;
    const R fn = fs - etaN * vn;
    const V3<R> vt = sub(vr, mul(nh, vn));
    xi = add(xi, mul(vt, dtt));
    xi = sub(xi, mul(nh, dot(xi, nh)));
    V3<R> ft = add(mul(xi, -st), mul(vt, -etaT));
    const R fl = std::sqrt(dot(ft, ft));
    const R fm = muE * std::fabs(fs);
    if (fl > fm) {
      const R s = (fl > R(1e-20)) ? fm / fl : R(0);
      ft = mul(ft, s);
      if (st > R(1e-20))
        xi = mul(add(ft, mul(vt, etaT)), R(-1) / st);
    }
    return add(mul(nh, fn), ft);
  }
  void pairEMu(int ma, int mb, R& e, R& f) const {
    if (!pairMat.empty()) {
      const int t = (ma * kMaxMaterials + mb) * 2;
      e = pairMat[t];
      f = pairMat[t + 1];
    } else {
      e = eN;
      f = mu;
    }
  }
  void stars(int ma, int mb, R& eS, R& gS) const {
    const R Ei = hzE[ma], Ej = hzE[mb], ni = hzNu[ma], nj = hzNu[mb];
    eS = R(1) / ((R(1) - ni * ni) / Ei + (R(1) - nj * nj) / Ej);
    gS = R(1) / (R(2) * (R(2) - ni) * (R(1) + ni) / Ei + R(2) * (R(2) - nj) * (R(1) + nj) / Ej);
  }
  // solver_hertz.hpp:88-144 (force/torque accumulation in ascending pair index)
  void hertzPairs(R dtt) {
    for (int idx = 0; idx < hzNumPairs; ++idx) {
      const int i = pairs[2 * idx], j = pairs[2 * idx + 1];
      const V3<R> dx = sub(pos[i], pos[j]);
      const R d = std::sqrt(dot(dx, dx));
      const R ri = rad[i], rj = rad[j];
      const R delta = ri + rj - d;
      if (delta <= R(0) || d < R(1e-12)) {
        hzXi[idx] = V3<R>{0, 0, 0};
        continue;
      }
      const V3<R> nh = mul(dx, R(1) / d);
      const V3<R> rA = mul(nh, -(ri - R(0.5) * delta));
      const V3<R> rB = mul(nh, (rj - R(0.5) * delta));
      const V3<R> vr = sub(add(vel[i], cross(angVel[i], rA)), add(vel[j], cross(angVel[j], rB)));
      const int ma = materialId[i], mb = materialId[j];
      R e, f, eS, gS;
      pairEMu(ma, mb, e, f);
      stars(ma, mb, eS, gS);
      const R rS = ri * rj / (ri + rj);
      const R imS = invMass[i] + invMass[j];
      const R mS = (imS > R(0)) ? R(1) / imS : R(0);
      V3<R> x = hzXi[idx];
      const V3<R> F = hertzForce(delta, nh, vr, rS, mS, eS, gS, e, f, dtt, x);
      hzXi[idx] = x;
      const V3<R> tA = cross(rA, F), tB = cross(rB, mul(F, R(-1)));
      deltaVel[i] = add(deltaVel[i], F);
      deltaVel[j] = add(deltaVel[j], neg(F));
      deltaAngVel[i] = add(deltaAngVel[i], tA);
      deltaAngVel[j] = add(deltaAngVel[j], tB);
    }
  }
  // solver_hertz.hpp:148-338 (spherical branch; shaped particles against walls below)
  void hertzWalls(R dtt, bool hasShapes) {
    const R* g = wallGrid.data();
    for (int ci = 0; ci < hzNumWallCand; ++ci) {
      const int enc = hzWallCand[ci];
      const int i = enc / 8, wi = enc % 8;
      const V3<R> p = pos[i];
      const R r = rad[i];
      const Wall<R>& w = walls[wi];
      const int slot = i * kHertzMaxWalls + wi;
      const int ma = materialId[i];
      R e, f;
      if (w.materialId >= 0 && !pairMat.empty())
        pairEMu(ma, w.materialId, e, f);
      else {
        e = w.restitution;
        f = w.friction;
      }
      const int mw = (w.materialId >= 0) ? w.materialId : ma;
      R eS, gS;
      stars(ma, mw, eS, gS);
      const R mS = (invMass[i] > R(0)) ? R(1) / invMass[i] : R(0);
      if (hasShapes && shapes[shapeId[i]].numPoints > 0) {
        const Shape<R>& dS = shapes[shapeId[i]];
        const V4<R> qP = quat[i];
        const R es = scale[i] * globalScale;
        const R rc = hzContactRadiusFrac * dS.par.x * es;
        const R bd = betaD(e);
        const V3<R> vP = vel[i], wP = angVel[i];
        const R snPrev = hzSnWall[slot];
        const R dampC = (mS > R(0)) ? R(-2) * R(0.9128709) * bd * std::sqrt(mS) : R(0);
        R fnSum = 0, snSum = 0, dMax = 0;
        V3<R> cSum{0, 0, 0}, nSum{0, 0, 0}, fAcc{0, 0, 0}, tAcc{0, 0, 0};
        for (int k = 0; k < dS.numPoints; ++k) {
          const V3<R> pW = add(p, rot(qP, mul(shell[dS.shellOffset + k], es)));
          const R sd = sampleWall(pW, w, g);
          if (sd >= R(0))
            continue;
          const R delta = -sd;
          const R hx = R(0.5) / w.invSpacing.x;
          V3<R> gr{(sampleWall(V3<R>{pW.x + hx, pW.y, pW.z}, w, g) - sampleWall(V3<R>{pW.x - hx, pW.y, pW.z}, w, g)),
                   (sampleWall(V3<R>{pW.x, pW.y + hx, pW.z}, w, g) - sampleWall(V3<R>{pW.x, pW.y - hx, pW.z}, w, g)),
                   (sampleWall(V3<R>{pW.x, pW.y, pW.z + hx}, w, g) - sampleWall(V3<R>{pW.x, pW.y, pW.z - hx}, w, g))};
          const R gl = len(gr);
          if (gl < R(1e-12))
            continue;
          const V3<R> nh = mul(gr, R(1) / gl);
          const V3<R> rA = sub(pW, p);
          const V3<R> vW = add(w.linVel, cross(w.angVel, sub(pW, w.center)));
          const V3<R> vrP = sub(add(vP, cross(wP, rA)), vW);
          const R vnP = dot(vrP, nh);
          const R sq = std::sqrt(rc * delta);
          const R fs = (R(4) / R(3)) * eS * sq * delta;
          const R snI = R(2) * eS * sq;
          const R snTot = (snPrev > snI) ? snPrev : snI;
          const R eta = dampC * snI / std::sqrt(snTot);
          const V3<R> F = mul(nh, fs - eta * vnP);
          fAcc = add(fAcc, F);
          tAcc = add(tAcc, cross(rA, F));
          fnSum += fs;
          snSum += R(2) * eS * sq;
          cSum = add(cSum, mul(pW, fs));
          nSum = add(nSum, mul(nh, fs));
          if (delta > dMax)
            dMax = delta;
        }
        if (fnSum <= R(0)) {
          hzXiWall[slot] = V3<R>{0, 0, 0};
          hzSnWall[slot] = 0;
          continue;
        }
        const V3<R> cpt = mul(cSum, R(1) / fnSum);
        V3<R> nh = nSum;
        const R nl = len(nh);
        if (nl > R(1e-9))
          nh = mul(nh, R(1) / nl);
        const V3<R> rA = sub(cpt, p);
        const V3<R> vW = add(w.linVel, cross(w.angVel, sub(cpt, w.center)));
        const V3<R> vr = sub(add(vP, cross(wP, rA)), vW);
        hzSnWall[slot] = snSum;
        const V3<R> vt = sub(vr, mul(nh, dot(vr, nh)));
        const R st = R(8) * gS * std::sqrt(rc * dMax);
        const R etaT = R(-2) * R(0.9128709) * bd * std::sqrt(st * mS);
        V3<R> x = hzXiWall[slot];
        x = add(x, mul(vt, dtt));
        x = sub(x, mul(nh, dot(x, nh)));
        V3<R> ft = add(mul(x, -st), mul(vt, -etaT));
        const R fl = len(ft);
        const R fm = f * fnSum;
        if (fl > fm) {
          const R s2 = (fl > R(1e-20)) ? fm / fl : R(0);
          ft = mul(ft, s2);
          if (st > R(1e-20))
            x = mul(add(ft, mul(vt, etaT)), R(-1) / st);
        }
        hzXiWall[slot] = x;
        fAcc = add(fAcc, ft);
        tAcc = add(tAcc, cross(rA, ft));
        deltaVel[i] = add(deltaVel[i], fAcc);
        deltaAngVel[i] = add(deltaAngVel[i], tAcc);
        continue;
      }
      const R s = sampleWall(p, w, g);
      const R delta = r - s;
      if (delta <= R(0)) {
        hzXiWall[slot] = V3<R>{0, 0, 0};
        continue;
      }
      const R hx = R(0.5) / w.invSpacing.x;
      V3<R> gr{(sampleWall(V3<R>{p.x + hx, p.y, p.z}, w, g) - sampleWall(V3<R>{p.x - hx, p.y, p.z}, w, g)),
               (sampleWall(V3<R>{p.x, p.y + hx, p.z}, w, g) - sampleWall(V3<R>{p.x, p.y - hx, p.z}, w, g)),
               (sampleWall(V3<R>{p.x, p.y, p.z + hx}, w, g) - sampleWall(V3<R>{p.x, p.y, p.z - hx}, w, g))};
      const R gl = std::sqrt(dot(gr, gr));
      if (gl < R(1e-12))
        continue;
      const V3<R> nh = mul(gr, R(1) / gl);
      const V3<R> rA = mul(nh, -(r - R(0.5) * delta));
      const V3<R> cpt = add(p, rA);
      const V3<R> vW = add(w.linVel, cross(w.angVel, sub(cpt, w.center)));
      const V3<R> vr = sub(add(vel[i], cross(angVel[i], rA)), vW);
      V3<R> x = hzXiWall[slot];
      const V3<R> F = hertzForce(delta, nh, vr, r, mS, eS, gS, e, f, dtt, x);
      hzXiWall[slot] = x;
      deltaVel[i] = add(deltaVel[i], F);
      deltaAngVel[i] = add(deltaAngVel[i], cross(rA, F));
    }
  }
  // solver_hertz.hpp:454-606 (point-shell pairs, one patch history per pair)
  void hertzShapePairs(R dtt) {
    for (int idx = 0; idx < hzNumPairs; ++idx) {
      const int A = pairs[2 * idx], B = pairs[2 * idx + 1];
      const Shape<R>& dA = shapes[shapeId[A]];
      const Shape<R>& dB = shapes[shapeId[B]];
      const V3<R> pA = pos[A], pB = pos[B];
      const V4<R> qA = quat[A], qB = quat[B];
      const R sA = scale[A] * globalScale, sB = scale[B] * globalScale;
      const int cnt = dA.numPoints;
      const bool sphA = dA.type == SPHERE;
      const int iter = cnt > 0 ? cnt : 1;
      const int ma = materialId[A], mb = materialId[B];
      R e, f, eS, gS;
      pairEMu(ma, mb, e, f);
      stars(ma, mb, eS, gS);
      const R rcA = (sphA ? R(1) : hzContactRadiusFrac) * dA.par.x * sA;
      const R rcB = ((dB.type == SPHERE) ? R(1) : hzContactRadiusFrac) * dB.par.x * sB;
      const R rS = rcA * rcB / (rcA + rcB);
      const R imS = invMass[A] + invMass[B];
      const R mS = (imS > R(0)) ? R(1) / imS : R(0);
      const R bd = betaD(e);
      const V3<R> vA = vel[A], wA = angVel[A], vB = vel[B], wB = angVel[B];
      R fnSum = 0, snSum = 0, dMax = 0;
      V3<R> cSum{0, 0, 0}, nSum{0, 0, 0}, fAcc{0, 0, 0}, tA{0, 0, 0}, tB{0, 0, 0};
      const R snPrev = hzSnPair[idx];
      const R dampC = (mS > R(0)) ? R(-2) * R(0.9128709) * bd * std::sqrt(mS) : R(0);
      for (int k = 0; k < iter; ++k) {
        V3<R> pl{0, 0, 0};
        R prad = 0;
        if (cnt > 0)
          pl = shell[dA.shellOffset + k];
        else if (sphA)
          prad = dA.par.x * sA;
        const V3<R> pw = add(pA, rot(qA, mul(pl, sA)));
        const V3<R> pc = mul(invrot(qB, sub(pw, pB)), R(1) / sB);
        const R dist = sdfShape(pc, dB, sdfGrid.data()) * sB;
        const R eff = dist - prad;
        if (eff >= R(0))
          continue;
        const R delta = -eff;
        const R eps = R(1e-4);
        V3<R> nl{sdfShape(V3<R>{pc.x + eps, pc.y, pc.z}, dB, sdfGrid.data()) -
                     sdfShape(V3<R>{pc.x - eps, pc.y, pc.z}, dB, sdfGrid.data()),
                 sdfShape(V3<R>{pc.x, pc.y + eps, pc.z}, dB, sdfGrid.data()) -
                     sdfShape(V3<R>{pc.x, pc.y - eps, pc.z}, dB, sdfGrid.data()),
                 sdfShape(V3<R>{pc.x, pc.y, pc.z + eps}, dB, sdfGrid.data()) -
                     sdfShape(V3<R>{pc.x, pc.y, pc.z - eps}, dB, sdfGrid.data())};
        const R l = len(nl);
        nl = (l > R(1e-9)) ? mul(nl, R(1) / l) : V3<R>{0, 1, 0};
        const V3<R> nW = rot(qB, nl);
        const V3<R> ps = sub(pw, mul(nW, prad));
        const V3<R> rA = sub(ps, pA);
        const V3<R> rB = sub(add(ps, mul(nW, delta)), pB);
        const V3<R> vrP = sub(add(vA, cross(wA, rA)), add(vB, cross(wB, rB)));
        const R vnP = dot(vrP, nW);
        const R sq = std::sqrt(rS * delta);
        const R fs = (R(4) / R(3)) * eS * sq * delta;
        const R snI = R(2) * eS * sq;
        const R snTot = (snPrev > snI) ? snPrev : snI;
        const R eta = dampC * snI / std::sqrt(snTot);
        const V3<R> F = mul(nW, fs - eta * vnP);
        fAcc = add(fAcc, F);
        tA = add(tA, cross(rA, F));
        tB = add(tB, cross(rB, mul(F, R(-1))));
        fnSum += fs;
        snSum += R(2) * eS * sq;
        cSum = add(cSum, mul(ps, fs));
        nSum = add(nSum, mul(nW, fs));
        if (delta > dMax)
          dMax = delta;
      }
      if (fnSum <= R(0)) {
        hzXi[idx] = V3<R>{0, 0, 0};
        hzSnPair[idx] = 0;
        continue;
      }
      const V3<R> cpt = mul(cSum, R(1) / fnSum);
      V3<R> nh = nSum;
      const R nl2 = len(nh);
      if (nl2 > R(1e-9))
        nh = mul(nh, R(1) / nl2);
      const V3<R> rA = sub(cpt, pA), rB = sub(cpt, pB);
      const V3<R> vr = sub(add(vA, cross(wA, rA)), add(vB, cross(wB, rB)));
      hzSnPair[idx] = snSum;
      const V3<R> vt = sub(vr, mul(nh, dot(vr, nh)));
      const R st = R(8) * gS * std::sqrt(rS * dMax);
      const R etaT = R(-2) * R(0.9128709) * bd * std::sqrt(st * mS);
      V3<R> x = hzXi[idx];
      x = add(x, mul(vt, dtt));
      x = sub(x, mul(nh, dot(x, nh)));
      V3<R> ft = add(mul(x, -st), mul(vt, -etaT));
      const R fl = len(ft);
      const R fm = f * fnSum;
      if (fl > fm) {
        const R s = (fl > R(1e-20)) ? fm / fl : R(0);
        ft = mul(ft, s);
        if (st > R(1e-20))
          x = mul(add(ft, mul(vt, etaT)), R(-1) / st);
      }
      hzXi[idx] = x;
      fAcc = add(fAcc, ft);
      tA = add(tA, cross(rA, ft));
      tB = add(tB, cross(rB, mul(ft, R(-1))));
      deltaVel[A] = add(deltaVel[A], fAcc);
      deltaVel[B] = add(deltaVel[B], neg(fAcc));
      deltaAngVel[A] = add(deltaAngVel[A], tA);
      deltaAngVel[B] = add(deltaAngVel[B], tB);
    }
  }
  // solver_hertz.hpp:374-425
  void hertzIntegrate(R dtt, bool orient) {
    for (int i = 0; i < numReal; ++i) {
      const R im = invMass[i];
      if (im > R(0)) {
        const V3<R> iI = invI[i];
        const V3<R> T = deltaAngVel[i];
        V3<R> dw;
        if (iI.x == iI.y && iI.y == iI.z) {
          dw = V3<R>{T.x * iI.x, T.y * iI.x, T.z * iI.x};
        } else {
          const V3<R> tl = invrot(quat[i], T);
          dw = rot(quat[i], V3<R>{tl.x * iI.x, tl.y * iI.y, tl.z * iI.z});
        }
        const V3<R> F = deltaVel[i];
        R* v = &vel[i].x;
        R* w = &angVel[i].x;
        R* x = &pos[i].x;
        const R* f = &F.x;
        const R* gg = &gravity.x;
        const R* d = &dw.x;
        for (int c = 0; c < 3; ++c) {
          v[c] += (f[c] * im + gg[c]) * dtt;
          w[c] += d[c] * dtt;
          x[c] += v[c] * dtt;
        }
        if (orient) {
          V4<R> q = quat[i];
          const V3<R> ww = angVel[i];
          const V4<R> dq{R(0.5) * dtt * (ww.x * q.w + ww.y * q.z - ww.z * q.y),
                         R(0.5) * dtt * (ww.y * q.w + ww.z * q.x - ww.x * q.z),
                         R(0.5) * dtt * (ww.z * q.w + ww.x * q.y - ww.y * q.x),
                         R(0.5) * dtt * (-ww.x * q.x - ww.y * q.y - ww.z * q.z)};
          q = V4<R>{q.x + dq.x, q.y + dq.y, q.z + dq.z, q.w + dq.w};
          const R qn = std::sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
          if (qn > R(1e-12))
            quat[i] = V4<R>{q.x / qn, q.y / qn, q.z / qn, q.w / qn};
        }
      }
      deltaVel[i] = V3<R>{0, 0, 0};
      deltaAngVel[i] = V3<R>{0, 0, 0};
    }
  }
  R hertzMaxDisp2() const {  // solver_hertz.hpp:429-444
    R m = std::numeric_limits<R>::lowest();
    for (int i = 0; i < numReal; ++i) {
      const V3<R> d = sub(pos[i], hzRefPos[i]);
      const R dd = dot(d, d);
      if (dd > m)
        m = dd;
    }
    return m;
  }
  void hertzCommitHistory() {  // sim.hpp:597-625
    const int n = hzNumPairs;
    if (n <= 0) {
      hzPrevCount = 0;
      return;
    }
    std::vector<int> perm(n);
    std::iota(perm.begin(), perm.end(), 0);
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return hzKeys[a] < hzKeys[b]; });
    for (int i = 0; i < n; ++i) {
      hzPrevKeys[i] = hzKeys[perm[i]];
      hzPrevXi[i] = hzXi[perm[i]];
    }
    hzPrevCount = n;
  }
  void hertzRebuildPairs(R skinW) {  // sim.hpp:545-594
    posPred = pos;
    const int np = findCollisionsGrow(skinW);
    const size_t need = (size_t)maxPairs;
    if (hzXi.size() < need) {
      hzXi.assign(need, V3<R>{0, 0, 0});
      hzSnPair.assign(need, R(0));
      hzKeys.assign(need, 0);
      hzPrevKeys.assign(need, 0);
      hzPrevXi.assign(need, V3<R>{0, 0, 0});
    }
    for (int idx = 0; idx < np; ++idx) {
      const unsigned a = (unsigned)pairs[2 * idx], b = (unsigned)pairs[2 * idx + 1];
      const unsigned lo = a < b ? a : b, hi = a < b ? b : a;
      const u64 k = ((u64)hi << 32) | lo;
      hzKeys[idx] = k;
      const int l = lowerBound(hzPrevKeys, hzPrevCount, k);
      const bool hit = l < hzPrevCount && hzPrevKeys[l] == k;
      hzXi[idx] = hit ? hzPrevXi[l] : V3<R>{0, 0, 0};
    }
    hzNumPairs = np;
    for (int i = 0; i < np; ++i)
      hzSnPair[i] = 0;
    for (int i = 0; i < numReal; ++i)
      hzRefPos[i] = pos[i];
  }
  int hertzWallCandidates(R skinW) {  // solver_hertz.hpp:343-370
    int cnt = 0;
    const int cap = (int)hzWallCand.size();
    for (int i = 0; i < numReal; ++i)
      for (int wi = 0; wi < (int)walls.size(); ++wi) {
        const R s = sampleWall(pos[i], walls[wi], wallGrid.data());
        if (s < rad[i] + skinW) {
          if (cnt < cap)
            hzWallCand[cnt] = i * 8 + wi;
          ++cnt;
        }
      }
    return cnt < cap ? cnt : cap;
  }
  void stepHertz(R dtt, int nsteps, R skinFrac) {  // sim.hpp:628-750
    dt = dtt;
    if (px || py || pz)
      throw std::runtime_error("step_hertz: periodic domains not supported");
    if (!planes.empty())
      throw std::runtime_error("step_hertz: analytic planes not supported (use an SDF wall)");
    if ((int)walls.size() > kHertzMaxWalls)
      throw std::runtime_error("step_hertz: too many SDF walls");
    for (int i = 0; i < numReal; ++i)
      rad[i] = scale[i] * globalScale * baseRadius;
    R minRad = std::numeric_limits<R>::max();
    for (int i = 0; i < numReal; ++i)
      if (rad[i] < minRad)
        minRad = rad[i];
    const R skinW = skinFrac * minRad;
    const R rebuildAt = R(0.25) * skinW * skinW;
    bool rebuild = hzNumPairs < 0;
    bool hasShapes = false;
    for (const auto& s : shapes)
      if (s.numPoints > 0)
        hasShapes = true;
    for (int k = 0; k < nsteps; ++k) {
      if (rebuild) {
        hertzCommitHistory();
        hertzRebuildPairs(skinW);
        if (!walls.empty())
          hzNumWallCand = hertzWallCandidates(skinW);
        rebuild = false;
      }
      if (hasShapes)
        hertzShapePairs(dtt);
      else
        hertzPairs(dtt);
      if (!walls.empty() && hzNumWallCand > 0)
        hertzWalls(dtt, hasShapes);
      hertzIntegrate(dtt, hasShapes);
      if ((k & 15) == 15 || k == nsteps - 1)
        if (hertzMaxDisp2() > rebuildAt)
          rebuild = true;
    }
    posPred = pos;
    velPred = vel;
  }
};

}  // namespace orc
