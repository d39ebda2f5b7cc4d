// Host orchestration of the B200 substep: facade setters/getters and the demStep stage sequence.
// Each stage names the reference function (file:line) it reproduces. All device work runs on the
// simulation's own stream; the host reads back only the counts that size the next stage (pair,
// contact, manifold totals and colouring progress).
#include <algorithm>
#include <cstring>
#include <numeric>

#include <cub/cub.cuh>

#include "pdem_broad.cuh"
#include "pdem_contact.cuh"
#include "pdem_hertz.cuh"
#include "pdem_kernels.cuh"
#include "pdem_multilevel.cuh"
#include "pdem_persist.cuh"
#include "pdem_radix.cuh"
#include "pdem_shell.hpp"
#include "pdem_sim.cuh"
#include "pdem_sdf.cuh"
#include "pdem_solve.cuh"

namespace pdem {

long gDeviceAllocs = 0;
static const int kOne = 1;  // H2D source of a device flag set from the host

void cudaCheck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    cudaGetLastError();  // a refused launch leaves its (non-sticky) error for the next check
    throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
  }
}
#define KCHECK(name) cudaCheck(cudaGetLastError(), name)

template <class R>
Sim<R>::Sim(int capacity) {
  cudaCheck(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  cudaCheck(cudaHostAlloc(reinterpret_cast<void**>(&pin_), kPinBytes, cudaHostAllocDefault), "pinned read-back block");
  {
    int dev = 0;
    cudaCheck(cudaGetDevice(&dev), "cudaGetDevice");
    cudaCheck(cudaDeviceGetAttribute(&numSMs_, cudaDevAttrMultiProcessorCount, dev), "SM count");
    int coop = 0;
    cudaCheck(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev), "cooperative launch attribute");
    if (!coop)
      throw CudaError("device does not support cooperative launches");
    // the growable buffers come from the default pool: keep what they free for their regrowth
    cudaMemPool_t pool;
    cudaCheck(cudaDeviceGetDefaultMemPool(&pool, dev), "default memory pool");
    uint64_t keep = UINT64_MAX;
    cudaCheck(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "pool release threshold");
  }
  for (int i = 0; i < 8; ++i) {
    hzE_[i] = R(1.0e9);
    hzNu_[i] = R(0.25);
  }
  ctr_.ensure(1, false, stream_);
  allocate(capacity, capacity * 64, capacity * 16);
  uploadHertzMaterials();
  initializeShape(SHAPE_SPHERE, R(1), R(0), R(0));
}
template <class R>
Sim<R>::~Sim() {
  if (stream_) {
    cudaStreamSynchronize(stream_);
    cudaStreamDestroy(stream_);
  }
  if (pin_)
    cudaFreeHost(pin_);
  if (tStart_) {
    cudaEventDestroy(tStart_);
    cudaEventDestroy(tStop_);
  }
  for (auto& pr : tuneEv_)
    for (auto& e : pr)
      if (e)
        cudaEventDestroy(e);
}

// src/particles.hpp:194-288
template <class R>
void Sim<R>::allocate(int cap, int mp, int mc) {
  capacity_ = cap;
  maxPairs_ = mp;
  for (auto* b : {&pos_, &vel_, &angVel_, &invI_, &posPred_, &velPred_, &angVelPred_, &quat_, &quatPred_,
                  &extF_, &dVel_, &dAngVel_, &dPos_})
    b->ensure(cap, false, stream_);
  for (auto* b : {&invMass_, &scale_, &target_, &rad_})
    b->ensure(cap, false, stream_);
  planeFric_.ensure(2 * (size_t)cap, false, stream_);
  for (auto* b : {&shapeId_, &realIdx_, &counts_})
    b->ensure(cap, false, stream_);
  grounded_.ensure(cap, false, stream_);
  matId_.ensure(cap, false, stream_);
  winner_.ensure(cap, false, stream_);
  mask_.ensure(cap, false, stream_);
  pairs_.ensure(mp, false, stream_);
  allocContactBuffers(mc);
  hzXiWall_.ensure((size_t)cap * kHertzMaxWalls, false, stream_);
  hzSnWall_.ensure((size_t)cap * kHertzMaxWalls, false, stream_);
  hzWallCand_.ensure((size_t)cap * 2, false, stream_);
  hzRefPos_.ensure(cap, false, stream_);
  hzED_.ensure(8, false, stream_);
  hzNuD_.ensure(8, false, stream_);
  refreshDev();
}
template <class R>
void Sim<R>::allocContactBuffers(int mc) {
  topoValid_ = false;
  maxContacts_ = mc;
  cab_.ensure(mc, false, stream_);
  for (auto* b : {&cn_, &crA_, &crB_, &cbv_})
    b->ensure(mc, false, stream_);
  for (auto* b : {&cColor_, &cSlot_, &mnp_, &mColor_})
    b->ensure(mc, false, stream_);
  posLamC_.ensure(mc, false, stream_);
  mab_.ensure(mc, false, stream_);
  for (auto* b : {&mN_, &mTA_, &mTB_, &mrA_, &mrB_, &mwv_, &lambdaT_, &prevLambdaT_, &vt0_})
    b->ensure(mc, false, stream_);
  pairKeys_.ensure(mc, false, stream_);
  prevKeys_.ensure(mc, false, stream_);
  persistent_.ensure(mc, false, stream_);
  sideFlags_.ensure(mc, false, stream_);
  for (auto* b : {&lambda_, &prevLambda_, &vn0_, &posImp_, &prevPosImp_})
    b->ensure(mc, false, stream_);
}
// src/particles.hpp:297-327 (matId grown too; the reference keeps it at the construction size)
template <class R>
void Sim<R>::ensureCapacity(int nc) {
  topoValid_ = false;
  if (nc <= capacity_)
    return;
  for (auto* b : {&pos_, &vel_, &angVel_, &invI_, &posPred_, &velPred_, &angVelPred_, &quat_, &quatPred_,
                  &extF_, &dVel_, &dAngVel_, &dPos_})
    b->ensure(nc, true, stream_);
  for (auto* b : {&invMass_, &scale_, &target_, &rad_})
    b->ensure(nc, true, stream_);
  planeFric_.ensure(2 * (size_t)nc, true, stream_);
  for (auto* b : {&shapeId_, &realIdx_, &counts_})
    b->ensure(nc, true, stream_);
  grounded_.ensure(nc, true, stream_);
  matId_.ensure(nc, true, stream_);
  winner_.ensure(nc, true, stream_);
  mask_.ensure(nc, true, stream_);
  capacity_ = nc;
  refreshDev();
}
// src/sim.hpp:1620-1654
template <class R>
void Sim<R>::ensureContactCapacity() {
  const int perParticle = std::max(16, shellPoints_);
  const long want = (long)capacity_ * perParticle + (long)capacity_ * std::max(1, shellPoints_) * wallsPerBody();
  if (want > maxContacts_) {
    allocContactBuffers((int)want);
    prevPairCount_ = 0;
    refreshDev();
  }
}
// walls a body can touch: all of them, or (batched form) the most that any one scene meets
template <class R>
long Sim<R>::wallsPerBody() const {
  if (!batch_)
    return (long)wallsHost_.size();
  long global = 0;
  std::vector<long> own(numScenes_, 0);
  for (size_t w = 0; w < wallsHost_.size(); ++w) {
    const int sc = w < wallScene_.size() ? wallScene_[w] : -1;
    if (sc < 0)
      ++global;
    else if (sc < numScenes_)
      ++own[sc];
  }
  return global + (own.empty() ? 0 : *std::max_element(own.begin(), own.end()));
}
template <class R>
void Sim<R>::refreshDev() {
  Dev<R>& d = d_;
  d.cap = capacity_;
  d.maxPairs = (int)pairs_.n;
  d.maxContacts = maxContacts_;
  d.pos = pos_.p, d.vel = vel_.p, d.angVel = angVel_.p, d.invI = invI_.p, d.posPred = posPred_.p;
  d.velPred = velPred_.p, d.angVelPred = angVelPred_.p, d.quat = quat_.p, d.quatPred = quatPred_.p;
  d.extForce = extF_.p, d.dVel = dVel_.p, d.dAngVel = dAngVel_.p, d.dPos = dPos_.p;
  d.invMass = invMass_.p, d.scale = scale_.p, d.targetScale = target_.p, d.rad = rad_.p;
  d.planeFric = planeFric_.p;
  d.shapeId = shapeId_.p, d.realIdx = realIdx_.p, d.counts = counts_.p;
  d.grounded = grounded_.p, d.matId = matId_.p, d.winner = winner_.p, d.mask = mask_.p;
  d.pairs = pairs_.p;
  d.cab = cab_.p, d.cn = cn_.p, d.crA = crA_.p, d.crB = crB_.p, d.cbv = cbv_.p;
  d.cColor = cColor_.p, d.cSlot = cSlot_.p, d.posLamC = posLamC_.p;
  d.mab = mab_.p, d.mnp = mnp_.p, d.mN = mN_.p, d.mTA = mTA_.p, d.mTB = mTB_.p, d.mrA = mrA_.p;
  d.mrB = mrB_.p, d.mwv = mwv_.p, d.mColor = mColor_.p;
  d.pairKeys = pairKeys_.p, d.prevKeys = prevKeys_.p, d.persistent = persistent_.p, d.sideFlags = sideFlags_.p;
  d.lambda = lambda_.p, d.prevLambda = prevLambda_.p, d.vn0 = vn0_.p, d.posImp = posImp_.p;
  d.prevPosImp = prevPosImp_.p, d.lambdaT = lambdaT_.p, d.prevLambdaT = prevLambdaT_.p, d.vt0 = vt0_.p;
  d.shapes = shapeD_.p, d.shell = shellD_.p, d.sdfGrid = sdfGridD_.p, d.planes = planesD_.p;
  d.walls = wallsD_.p, d.wallGrid = wallGridD_.p;
  d.pairMat = pairMatHost_.empty() ? nullptr : pairMatD_.p;
  d.hzE = hzED_.p, d.hzNu = hzNuD_.p;
  d.ctr = ctr_.p;
  d.numScenes = batch_ ? numScenes_ : 1;
  d.sceneOf = batch_ ? sceneOf_.p : nullptr;
  d.scn = batch_ ? scn_.p : nullptr;
  d.sceneWallOff = batch_ ? sceneWallOffD_.p : nullptr;
  d.sceneWallIdx = batch_ ? sceneWallIdxD_.p : nullptr;
  d.sceneManFirst = batch_ ? sceneManFirstD_.p : nullptr;
  d.sceneConFirst = batch_ ? sceneConFirstD_.p : nullptr;
  d.sceneLeafFirst = batch_ ? sceneLeafFirstD_.p : nullptr;
}
template <class R>
void Sim<R>::sync() {
  cudaCheck(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
  for (const PendingRead& r : pending_)
    std::memcpy(r.host, pin_ + r.off, r.bytes);
  dropPending();
}
template <class R>
void Sim<R>::readBack(void* host, const void* dev, size_t bytes) {
  const size_t off = (pinOff_ + 15) & ~size_t(15);
  if (!pin_ || off + bytes > kPinBytes) {  // no room: a direct copy, complete when it returns
    cudaCheck(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, stream_), "D2H");
    return;
  }
  cudaCheck(cudaMemcpyAsync(pin_ + off, dev, bytes, cudaMemcpyDeviceToHost, stream_), "D2H");
  pending_.push_back({host, off, bytes});
  pinOff_ = off + bytes;
}
// a timed-out barrier has been reported: clear its error bit so the next substep starts clean (the
// barrier words are zeroed before every cooperative launch)
template <class R>
void Sim<R>::clearLoopError() {
  dropPending();
  cudaCheck(cudaMemsetAsync(&ctr_.p->err, 0, sizeof(int), stream_), "memset error bits");
  sync();
}
template <class R>
Counters<R> Sim<R>::readCounters() {
  Counters<R> c;
  readBack(&c, ctr_.p, sizeof c);
  sync();
  if (c.err & kErrBarrier) {
    clearLoopError();
    throw CudaError("a grid-wide barrier of a persistent loop timed out (blocks not co-resident)");
  }
  return c;
}

// blocks of a cooperative launch of `kernel`: resident blocks per SM (at most 4) x SMs, the
// occupancy query cached by (kernel, block). A grid sized down to a small scene's work was not
// faster: a colour step there is bound by the latency of one PGS update, not by the barrier.
template <class R>
template <class K>
int Sim<R>::coopGrid(K kernel, int block) {
  const auto key = std::make_pair(reinterpret_cast<const void*>(kernel), block);
  auto it = coopPer_.find(key);
  if (it == coopPer_.end()) {
    int per = 0;
    cudaCheck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, block, 0), "occupancy");
    if (per < 1)
      throw CudaError("persistent loop kernel cannot be resident");
    it = coopPer_.emplace(key, per).first;
  }
  return std::min(it->second, 4) * numSMs_;
}
template <class R>
template <class K, class... A>
void Sim<R>::launchCoopB(K kernel, int block, A... args) {
  gbar_.ensure(2, false, stream_);
  cudaCheck(cudaMemsetAsync(gbar_.p, 0, 2 * sizeof(unsigned), stream_), "memset barrier");
  void* argv[] = {static_cast<void*>(&args)...};
  ++launches_;
  cudaCheck(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kernel), dim3(coopGrid(kernel, block)),
                                        dim3(block), argv, 0, stream_),
            "cooperative launch");
}
template <class R>
template <class K, class... A>
void Sim<R>::launchCoop(K kernel, A... args) {
  launchCoopB(kernel, kBlock, args...);
}
template <class R>
template <class K, class... A>
void Sim<R>::launchCoopSmem(K kernel, int block, size_t smem, A... args) {
  const auto key = std::make_tuple(reinterpret_cast<const void*>(kernel), block, smem);
  auto it = coopPerSmem_.find(key);
  if (it == coopPerSmem_.end()) {
    cudaCheck(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem attribute");
    int per = 0;
    cudaCheck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, block, smem), "occupancy");
    if (per < 1)
      throw CudaError("persistent loop kernel cannot be resident");
    it = coopPerSmem_.emplace(key, per).first;
  }
  gbar_.ensure(2, false, stream_);
  cudaCheck(cudaMemsetAsync(gbar_.p, 0, 2 * sizeof(unsigned), stream_), "memset barrier");
  void* argv[] = {static_cast<void*>(&args)...};
  ++launches_;
  cudaCheck(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kernel), dim3(std::min(it->second, 4) * numSMs_),
                                        dim3(block), argv, smem, stream_),
            "cooperative launch");
}
template <class R>
template <class K, class... A>
bool Sim<R>::launchCluster(K kernel, A... args) {
  return launchClusterCfg(kernel, sweepClusterBlocks_, kBlock, 0, args...);
}
template <class R>
template <class K, class... A>
bool Sim<R>::launchClusterCfg(K kernel, int blocks, int block, size_t smem, A... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream_;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = blocks;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const void* key = reinterpret_cast<const void*>(kernel);
  auto it = clusterOk_.find(key);
  if (it == clusterOk_.end()) {
    int clusters = 0;
    if (blocks > 8 && cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
      (void)cudaGetLastError();
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      (void)cudaGetLastError();
    if (cudaOccupancyMaxActiveClusters(&clusters, kernel, &cfg) != cudaSuccess)
      (void)cudaGetLastError();
    it = clusterOk_.emplace(key, clusters >= 1 ? 1 : 0).first;
  }
  if (!it->second)
    return false;
  ++launches_;
  cudaCheck(cudaLaunchKernelEx(&cfg, kernel, args...), "cluster launch");
  return true;
}

// the colour-ordered velocity-sweep records of this substep's manifolds, packed at the first
// request of a substep (the orientations and masses they hold do not change until the
// integration after the stabilization pass)
template <class R>
PgsRecs<R> Sim<R>::packPgs(int nm, int ncol) {
  if (pgsPackedAt_ != substepId_) {
    // the slot stride is the ids' capacity, so the slots are sized from it after it grew
    pgsIds_.ensure((size_t)nm, false, stream_);
    pgsCap_ = (long)(pgsIds_.n);
    pgsQ_.ensure((size_t)kPgsSlots * pgsIds_.n, false, stream_);
    ++launches_, kPackPgs<R><<<gridFor(nm), kBlock, 0, stream_>>>(d_, mOrder_.p, mOff_.p, ncol,
                                                                 PgsRecs<R>{pgsQ_.p, pgsIds_.p, pgsCap_});
    KCHECK("pack velocity records");
    pgsPackedAt_ = substepId_;
  }
  return PgsRecs<R>{pgsQ_.p, pgsIds_.p, pgsCap_};
}

// ---- CUB helpers ----
template <class R>
template <class T>
void Sim<R>::sortPairs(const T* kin, T* kout, const int* vin, int* vout, int n, int endBit) {
  if (n <= 0)
    return;
  size_t bytes = 0;
  cudaCheck(cub::DeviceRadixSort::SortPairs(nullptr, bytes, kin, kout, vin, vout, n, 0, endBit, stream_), "cub sort");
  cubTmp_.ensure(bytes, false, stream_);
  cudaCheck(cub::DeviceRadixSort::SortPairs(cubTmp_.p, bytes, kin, kout, vin, vout, n, 0, endBit, stream_), "cub sort");
}
template <class R>
template <class T>
void Sim<R>::exclusiveSum(const T* in, T* out, int n) {
  size_t bytes = 0;
  cudaCheck(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, stream_), "cub scan");
  cubTmp_.ensure(bytes, false, stream_);
  cudaCheck(cub::DeviceScan::ExclusiveSum(cubTmp_.p, bytes, in, out, n, stream_), "cub scan");
}
template <class R>
template <class T>
void Sim<R>::inclusiveSum(const T* in, T* out, int n) {
  size_t bytes = 0;
  cudaCheck(cub::DeviceScan::InclusiveSum(nullptr, bytes, in, out, n, stream_), "cub scan");
  cubTmp_.ensure(bytes, false, stream_);
  cudaCheck(cub::DeviceScan::InclusiveSum(cubTmp_.p, bytes, in, out, n, stream_), "cub scan");
}
static int bitsFor(long maxValue) {
  int b = 1;
  while (b < 64 && (1L << b) <= maxValue)
    ++b;
  return b;
}

// =============================================================================================
// facade setters (src/sim.hpp:943-1424)
// =============================================================================================
// src/sim.hpp:949-1021
template <class R>
void Sim<R>::initializeShape(int type, R radius, R height, R thick) {
  vValid_ = false;  // box sizes, parking or images may change
  baseRadius_ = radius;
  ShapeDesc<R> sd{};
  std::vector<ShellPoint> sh;
  if (type == SHAPE_HCYL) {
    sd.par[0] = radius, sd.par[1] = height, sd.par[2] = thick, sd.par[3] = 0;
    const float rf = (float)radius, tf = (float)thick;
    float minDim = std::min(rf, tf);
    if (minDim < 1e-4f)
      minDim = rf;
    float sp = std::min(rf * 0.3f, minDim * 0.5f);
    if (sp < 1e-3f)
      sp = 1e-3f;
    sh = hollowCylinderShell(rf, (float)height, tf, sp);
  } else if (type == SHAPE_BOX) {
    sd.par[0] = sd.par[1] = sd.par[2] = radius;
    const float sp = std::max((float)radius * 0.5f, 1e-3f);
    sh = boxShell((float)radius, (float)radius, (float)radius, sp);
  } else {
    type = SHAPE_SPHERE;
    sd.par[0] = radius;
  }
  const int n = (int)sh.size();
  shellPoints_ = n;
  if (n > 0) {
    shellHost_.resize(n);
    for (int i = 0; i < n; ++i)
      shellHost_[i] = Q4<R>{R(sh[i].x), R(sh[i].y), R(sh[i].z), R(0)};
  }
  sd.type = type;
  sd.numPoints = n;
  sd.shellOffset = 0;
  shape_ = sd;
  uploadShape();
  R ix = 1, iy = 1, iz = 1;
  if (type == SHAPE_SPHERE) {
    if (baseRadius_ > R(0)) {
      const R v = R(2.5) / (baseRadius_ * baseRadius_);
      ix = iy = iz = v;
    }
  } else if (type == SHAPE_HCYL) {
    const R ro = baseRadius_;
    R ri = baseRadius_ - thick;
    if (ri < 0)
      ri = 0;
    const R tr = ro * ro + ri * ri;
    const R Izz = R(0.5) * tr;
    const R Ixx = (R(1.0) / R(12.0)) * (R(3.0) * tr + height * height);
    if (Ixx > R(1e-6))
      ix = iy = R(1.0) / Ixx;
    if (Izz > R(1e-6))
      iz = R(1.0) / Izz;
  } else if (type == SHAPE_BOX) {
    const R L = R(2.0) * baseRadius_;
    const R I = (R(1.0) / R(6.0)) * L * L;
    if (I > R(1e-6))
      ix = iy = iz = R(1.0) / I;
  }
  defInvI_[0] = ix, defInvI_[1] = iy, defInvI_[2] = iz;
}
template <class R>
void Sim<R>::uploadShape() {
  double r2 = 0;
  for (int k = 0; k < shape_.numPoints && k < (int)shellHost_.size(); ++k) {
    const Q4<R>& q = shellHost_[k];
    r2 = std::max(r2, (double)q.x * q.x + (double)q.y * q.y + (double)q.z * q.z);
  }
  shape_.shellR = std::nextafter((R)std::sqrt(r2), std::numeric_limits<R>::infinity());
  shapeD_.ensure(1, false, stream_);
  cudaCheck(cudaMemcpyAsync(shapeD_.p, &shape_, sizeof shape_, cudaMemcpyHostToDevice, stream_), "H2D shape");
  const size_t ns = std::max<size_t>(1, shellHost_.size());
  shellD_.ensure(ns, false, stream_);
  if (!shellHost_.empty())
    cudaCheck(cudaMemcpyAsync(shellD_.p, shellHost_.data(), shellHost_.size() * sizeof(Q4<R>),
                              cudaMemcpyHostToDevice, stream_), "H2D shell");
  sdfGridD_.ensure(std::max<size_t>(1, sdfGridHost_.size()), false, stream_);
  if (!sdfGridHost_.empty())
    cudaCheck(cudaMemcpyAsync(sdfGridD_.p, sdfGridHost_.data(), sdfGridHost_.size() * sizeof(R),
                              cudaMemcpyHostToDevice, stream_), "H2D sdf grid");
  sync();
  refreshDev();
}
template <class R>
void Sim<R>::setShellPoints(const std::vector<R>& p) {
  vValid_ = false;  // box sizes, parking or images may change
  const int n = (int)(p.size() / 3);
  shellHost_.assign(std::max(n, 1), Q4<R>{0, 0, 0, 0});
  for (int i = 0; i < n; ++i)
    shellHost_[i] = Q4<R>{p[3 * i], p[3 * i + 1], p[3 * i + 2], R(0)};
  if (n == 0)
    shellHost_.clear();
  shape_.numPoints = n;
  shape_.shellOffset = 0;
  shellPoints_ = n;
  uploadShape();
  ensureContactCapacity();
}
// src/sim.hpp:1034-1084
template <class R>
void Sim<R>::setSdfShape(const std::vector<R>& grid, int nx, int ny, int nz, const R* origin, const R* spacing,
                         const std::vector<R>& shell, const R* invI, R bR) {
  vValid_ = false;  // box sizes, parking or images may change
  if (nx < 2 || ny < 2 || nz < 2)
    throw std::runtime_error("setSdfShape: grid dims must be >= 2 on each axis");
  if ((long)nx * ny * nz != (long)grid.size())
    throw std::runtime_error("setSdfShape: grid.size() must equal nx*ny*nz");
  const int n = (int)(shell.size() / 3);
  if (n <= 0)
    throw std::runtime_error("setSdfShape: empty surface point shell");
  sdfGridHost_ = grid;
  shellHost_.resize(n);
  for (int i = 0; i < n; ++i)
    shellHost_[i] = Q4<R>{shell[3 * i], shell[3 * i + 1], shell[3 * i + 2], R(0)};
  ShapeDesc<R> sd{};
  sd.type = SHAPE_GRID;
  sd.par[0] = bR;
  sd.numPoints = n;
  sd.nx = nx, sd.ny = ny, sd.nz = nz;
  for (int a = 0; a < 3; ++a) {
    sd.gridOrigin[a] = origin[a];
    sd.gridInvSpacing[a] = spacing[a] > 0 ? R(1) / spacing[a] : R(0);
  }
  shape_ = sd;
  baseRadius_ = bR;
  defInvI_[0] = invI[0], defInvI_[1] = invI[1], defInvI_[2] = invI[2];
  shellPoints_ = n;
  uploadShape();
  ensureContactCapacity();
}
template <class R>
void Sim<R>::setDomain(R lx, R ly, R lz, bool px, bool py, bool pz) {
  vValid_ = false;  // box sizes, parking or images may change
  dmin_[0] = dmin_[1] = dmin_[2] = 0;
  dmax_[0] = dsize_[0] = lx;
  dmax_[1] = dsize_[1] = ly;
  dmax_[2] = dsize_[2] = lz;
  per_[0] = px, per_[1] = py, per_[2] = pz;
  skin_ = R(0.1) * gs_;
}
template <class R>
void Sim<R>::setDomainMinMax(const R* mn, const R* mx) {
  vValid_ = false;  // box sizes, parking or images may change
  for (int a = 0; a < 3; ++a) {
    dmin_[a] = mn[a];
    dmax_[a] = mx[a];
    dsize_[a] = mx[a] - mn[a];
  }
  skin_ = R(0.1) * gs_;
}
template <class R>
void Sim<R>::enablePeriodicity(bool x, bool y, bool z) {
  vValid_ = false;  // box sizes, parking or images may change
  per_[0] = x, per_[1] = y, per_[2] = z;
}
template <class R>
void Sim<R>::setStabilizationMode(const std::string& m) {
  if (m == "off")
    stabMode_ = 0;
  else if (m == "onesided")
    stabMode_ = 1;
  else if (m == "multilevel")
    stabMode_ = 2;
  else if (m == "escalate")
    stabMode_ = 3;
  else if (m == "ordered")
    stabMode_ = 4;
  else
    throw std::invalid_argument(
        "set_stabilization_mode: expected 'off', 'onesided', 'multilevel', 'escalate' or 'ordered'");
}
template <class R>
void Sim<R>::setHertzMaterial(int mat, R E, R nu) {
  if (mat < 0 || mat >= 8)
    throw std::invalid_argument("material id out of range");
  hzE_[mat] = E;
  hzNu_[mat] = nu;
  uploadHertzMaterials();
}
template <class R>
void Sim<R>::uploadHertzMaterials() {
  cudaCheck(cudaMemcpyAsync(hzED_.p, hzE_, sizeof hzE_, cudaMemcpyHostToDevice, stream_), "H2D hertz E");
  cudaCheck(cudaMemcpyAsync(hzNuD_.p, hzNu_, sizeof hzNu_, cudaMemcpyHostToDevice, stream_), "H2D hertz nu");
  sync();
}
template <class R>
void Sim<R>::setMaterialIds(const int* ids, int n) {
  const int m = std::min(numReal_, n);
  if (m <= 0)
    return;
  std::vector<uint8_t> h(m);
  for (int i = 0; i < m; ++i)
    h[i] = (uint8_t)ids[i];
  cudaCheck(cudaMemcpyAsync(matId_.p, h.data(), m, cudaMemcpyHostToDevice, stream_), "H2D matId");
  sync();
}
// src/sim.hpp:1196-1216
template <class R>
void Sim<R>::setPairMaterial(int a, int b, R e, R f) {
  if (a < 0 || b < 0 || a >= kMaxMaterials || b >= kMaxMaterials)
    throw std::invalid_argument("material id out of range");
  if (pairMatHost_.empty()) {
    pairMatHost_.assign(kMaxMaterials * kMaxMaterials * 2, R(0));
    for (int i = 0; i < kMaxMaterials * kMaxMaterials; ++i) {
      pairMatHost_[2 * i] = eN_;
      pairMatHost_[2 * i + 1] = mu_;
    }
  }
  pairMatHost_[(a * kMaxMaterials + b) * 2] = e;
  pairMatHost_[(a * kMaxMaterials + b) * 2 + 1] = f;
  pairMatHost_[(b * kMaxMaterials + a) * 2] = e;
  pairMatHost_[(b * kMaxMaterials + a) * 2 + 1] = f;
  pairMatD_.ensure(pairMatHost_.size(), false, stream_);
  cudaCheck(cudaMemcpyAsync(pairMatD_.p, pairMatHost_.data(), pairMatHost_.size() * sizeof(R),
                            cudaMemcpyHostToDevice, stream_), "H2D pair table");
  sync();
  refreshDev();
}
template <class R>
void Sim<R>::setWallMaterialId(int wid, int mat) {
  if (wid < 0 || wid >= (int)wallsHost_.size())
    throw std::invalid_argument("wall index out of range");
  wallsHost_[wid].materialId = mat;
  uploadWalls();
}
template <class R>
void Sim<R>::addPlane(const R* p, const R* n) {
  if ((int)planesHost_.size() < kMaxPlanes) {
    PlaneDesc<R> pl;
    for (int a = 0; a < 3; ++a) {
      pl.p[a] = p[a];
      pl.n[a] = n[a];
    }
    planesHost_.push_back(pl);
  }
  planesD_.ensure(kMaxPlanes, false, stream_);
  cudaCheck(cudaMemcpyAsync(planesD_.p, planesHost_.data(), planesHost_.size() * sizeof(PlaneDesc<R>),
                            cudaMemcpyHostToDevice, stream_), "H2D planes");
  sync();
  refreshDev();
}
// src/sim.hpp:1242-1274
template <class R>
int Sim<R>::addSdfWall(const std::vector<R>& grid, int nx, int ny, int nz, const R* origin, const R* spacing, R e,
                       R f) {
  if (nx < 2 || ny < 2 || nz < 2)
    throw std::runtime_error("addSdfWall: grid dims must be >= 2 on each axis");
  if ((long)nx * ny * nz != (long)grid.size())
    throw std::runtime_error("addSdfWall: grid.size() must equal nx*ny*nz");
  WallDesc<R> w{};
  w.nx = nx, w.ny = ny, w.nz = nz;
  // a grid identical to one already held (the same container in many batched scenes) is shared
  int shared = -1;
  for (const WallDesc<R>& o : wallsHost_)
    if (o.nx == nx && o.ny == ny && o.nz == nz &&
        std::equal(grid.begin(), grid.end(), wallGridHost_.begin() + o.gridOffset)) {
      shared = o.gridOffset;
      break;
    }
  w.gridOffset = shared >= 0 ? shared : (int)wallGridHost_.size();
  for (int a = 0; a < 3; ++a) {
    w.origin[a] = origin[a];
    w.invSpacing[a] = spacing[a] > 0 ? R(1) / spacing[a] : R(0);
  }
  w.restitution = e;
  w.friction = f;
  w.materialId = -1;
  wallsHost_.push_back(w);
  if (shared < 0) {
    wallGridHost_.insert(wallGridHost_.end(), grid.begin(), grid.end());
    wallGridD_.ensure(wallGridHost_.size(), false, stream_);
    cudaCheck(cudaMemcpyAsync(wallGridD_.p, wallGridHost_.data(), wallGridHost_.size() * sizeof(R),
                              cudaMemcpyHostToDevice, stream_), "H2D wall grid");
  }
  wallScene_.resize(wallsHost_.size(), -1);
  sceneWallsDirty_ = true;
  uploadWalls();
  if (f > wallFrictionMax_)
    wallFrictionMax_ = f;
  ensureContactCapacity();
  return (int)wallsHost_.size() - 1;
}
template <class R>
void Sim<R>::uploadWalls() {
  wallsD_.ensure(std::max<size_t>(1, wallsHost_.size()), false, stream_);
  if (!wallsHost_.empty())
    cudaCheck(cudaMemcpyAsync(wallsD_.p, wallsHost_.data(), wallsHost_.size() * sizeof(WallDesc<R>),
                              cudaMemcpyHostToDevice, stream_), "H2D walls");
  sync();
  refreshDev();
}
template <class R>
void Sim<R>::setWallVelocity(int idx, const R* lin, const R* ang, const R* center) {
  if (idx < 0 || idx >= (int)wallsHost_.size())
    throw std::runtime_error("setWallVelocity: wall index out of range");
  for (int a = 0; a < 3; ++a) {
    wallsHost_[idx].linVel[a] = lin[a];
    wallsHost_[idx].angVel[a] = ang[a];
    wallsHost_[idx].center[a] = center[a];
  }
  uploadWalls();
}
// src/sim.hpp:1290-1330
template <class R>
void Sim<R>::setPositions(const R* xyz, int n) {
  if (n > capacity_)
    throw std::invalid_argument("set_positions: more particles than the simulation capacity");
  ensureGrounded();  // the logged support graphs index the previous particle set
  if (batch_ && n != numReal_)
    batch_ = false;  // the scene layout described the previous particle set
  sceneParamsDirty_ = true;
  maxScaleValid_ = false;
  vValid_ = false;
  bvhValid_ = false;
  topoValid_ = false;
  numReal_ = n;
  numParticles_ = n;
  hzNumPairs_ = -1;
  hzPrevCount_ = 0;
  std::vector<Q4<R>> p(n), q(n, Q4<R>{0, 0, 0, 1}), ii(n, Q4<R>{defInvI_[0], defInvI_[1], defInvI_[2], 0}),
      z(n, Q4<R>{0, 0, 0, 0});
  std::vector<R> ones(n, R(1));
  std::vector<int> zi(n, 0);
  for (int i = 0; i < n; ++i)
    p[i] = Q4<R>{xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], R(0)};
  auto up = [&](void* dst, const void* src, size_t bytes) {
    if (bytes)
      cudaCheck(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream_), "H2D state");
  };
  up(pos_.p, p.data(), n * sizeof(Q4<R>));
  up(quat_.p, q.data(), n * sizeof(Q4<R>));
  up(invMass_.p, ones.data(), n * sizeof(R));
  up(scale_.p, ones.data(), n * sizeof(R));
  up(shapeId_.p, zi.data(), n * sizeof(int));
  up(invI_.p, ii.data(), n * sizeof(Q4<R>));
  up(vel_.p, z.data(), n * sizeof(Q4<R>));
  up(angVel_.p, z.data(), n * sizeof(Q4<R>));
  cudaCheck(cudaMemcpyAsync(target_.p, scale_.p, capacity_ * sizeof(R), cudaMemcpyDeviceToDevice, stream_), "D2D");
  sync();
}
// field codes: 0 vel, 1 extForce, 2 quat, 3 angVel, 4 invI, 5 invMass
template <class R>
void Sim<R>::setRows(int field, const R* a, int n) {
  const int m = std::min(numReal_, n);
  if (m <= 0)
    return;
  if (field == 5) {
    cudaCheck(cudaMemcpyAsync(invMass_.p, a, m * sizeof(R), cudaMemcpyHostToDevice, stream_), "H2D invMass");
    sync();
    return;
  }
  std::vector<Q4<R>> h(m);
  const int cols = (field == 2) ? 4 : 3;
  for (int i = 0; i < m; ++i)
    h[i] = Q4<R>{a[cols * i], a[cols * i + 1], a[cols * i + 2], cols == 4 ? a[cols * i + 3] : R(0)};
  Q4<R>* dst = field == 0 ? vel_.p : field == 1 ? extF_.p : field == 2 ? quat_.p : field == 3 ? angVel_.p : invI_.p;
  cudaCheck(cudaMemcpyAsync(dst, h.data(), m * sizeof(Q4<R>), cudaMemcpyHostToDevice, stream_), "H2D rows");
  sync();
}
// rows of a 4-wide field straight from the caller's doubles: one copy to the device, packed
// there (fields as setRows: 0 velocities, 1 external forces, 2 quaternions, 3 angular
// velocities, 4 inverse inertia)
template <class R>
void Sim<R>::setRowsD(int field, const double* a, int n) {
  const int m = std::min(numReal_, n);
  if (m <= 0)
    return;
  const int cols = (field == 2) ? 4 : 3;
  rowStage_.ensure((size_t)m * cols, false, stream_);
  cudaCheck(cudaMemcpyAsync(rowStage_.p, a, (size_t)m * cols * sizeof(double), cudaMemcpyHostToDevice, stream_),
            "H2D rows");
  Q4<R>* dst = field == 0 ? vel_.p : field == 1 ? extF_.p : field == 2 ? quat_.p : field == 3 ? angVel_.p : invI_.p;
  ++launches_, kPackRows<R><<<gridFor(m), kBlock, 0, stream_>>>(rowStage_.p, m, cols, dst);
  KCHECK("pack rows");
  sync();
}
// rows of a 4-wide field to the caller's doubles (fields as getRows: 0 positions, 1 velocities,
// 2 quaternions, 3 angular velocities, 4 inverse inertia): unpacked on the device, one copy back
template <class R>
void Sim<R>::getRowsD(int field, double* out, long cap) {
  const int n = numReal_;
  if (n <= 0)
    return;
  const int cols = (field == 2) ? 4 : 3;
  const long need = (long)n * cols;
  rowStage_.ensure(need, false, stream_);
  const Q4<R>* src = field == 0 ? pos_.p : field == 1 ? vel_.p : field == 2 ? quat_.p : field == 3 ? angVel_.p : invI_.p;
  ++launches_, kUnpackRows<R><<<gridFor(n), kBlock, 0, stream_>>>(src, n, cols, rowStage_.p);
  KCHECK("unpack rows");
  if (cap >= need) {
    cudaCheck(cudaMemcpyAsync(out, rowStage_.p, need * sizeof(double), cudaMemcpyDeviceToHost, stream_), "D2H rows");
    sync();
  } else {
    std::vector<double> h(need);
    cudaCheck(cudaMemcpyAsync(h.data(), rowStage_.p, need * sizeof(double), cudaMemcpyDeviceToHost, stream_),
              "D2H rows");
    sync();
    std::copy(h.begin(), h.begin() + std::max(cap, 0L), out);
  }
}
template <class R>
void Sim<R>::clearExternalForces() {
  extF_.zero(stream_);
  sync();
}
template <class R>
void Sim<R>::setScales(const R* s, int n) {  // src/sim.hpp:1340-1346
  sceneParamsDirty_ = true;
  maxScaleValid_ = false;
  vValid_ = false;
  const int m = std::min(numReal_, n);
  if (m > 0)
    cudaCheck(cudaMemcpyAsync(target_.p, s, m * sizeof(R), cudaMemcpyHostToDevice, stream_), "H2D scales");
  cudaCheck(cudaMemcpyAsync(scale_.p, target_.p, capacity_ * sizeof(R), cudaMemcpyDeviceToDevice, stream_), "D2D");
  sync();
}
template <class R>
void Sim<R>::setScalesUniform(R s) {  // src/sim.hpp:1331-1337
  sceneParamsDirty_ = true;
  maxScaleValid_ = false;
  vValid_ = false;
  if (numReal_ > 0) {
    std::vector<R> h(numReal_, s);
    cudaCheck(cudaMemcpyAsync(scale_.p, h.data(), numReal_ * sizeof(R), cudaMemcpyHostToDevice, stream_), "H2D");
  }
  cudaCheck(cudaMemcpyAsync(target_.p, scale_.p, capacity_ * sizeof(R), cudaMemcpyDeviceToDevice, stream_), "D2D");
  sync();
}
template <class R>
void Sim<R>::setGrowthParams(R rate, R nf) {  // src/sim.hpp:1416-1424
  if (gf_ == R(-1))
    gf_ = (nf > R(0)) ? nf : R(0.01);
  else if (nf > R(0))
    gf_ = nf;
  gr_ = rate;
  maxScaleValid_ = false;
  vValid_ = false;
  if (gf_ > R(0) && numReal_ > 0) {
    ++launches_, kGrowthScales<<<gridFor(numReal_), kBlock, 0, stream_>>>(d_, numReal_, gf_);
    KCHECK("growth");
    sync();
  }
}
// field codes: 0 pos, 1 vel, 2 quat, 3 angVel, 4 invI, 5 scale, 6 masses
template <class R>
void Sim<R>::getRows(int field, R* out, long cap) {
  const int n = numReal_;
  if (n <= 0)
    return;
  if (field >= 5) {
    std::vector<R> h(n);
    cudaCheck(cudaMemcpyAsync(h.data(), field == 5 ? scale_.p : invMass_.p, n * sizeof(R), cudaMemcpyDeviceToHost,
                              stream_), "D2H");
    sync();
    for (int i = 0; i < n && i < cap; ++i)
      out[i] = (field == 5) ? h[i] : ((h[i] > R(0)) ? R(1) / h[i] : R(0));
    return;
  }
  std::vector<Q4<R>> h(n);
  const Q4<R>* src = field == 0 ? pos_.p : field == 1 ? vel_.p : field == 2 ? quat_.p : field == 3 ? angVel_.p : invI_.p;
  cudaCheck(cudaMemcpyAsync(h.data(), src, n * sizeof(Q4<R>), cudaMemcpyDeviceToHost, stream_), "D2H rows");
  sync();
  const int cols = (field == 2) ? 4 : 3;
  for (int i = 0; i < n && (long)cols * i + cols - 1 < cap; ++i) {
    out[cols * i] = h[i].x;
    out[cols * i + 1] = h[i].y;
    out[cols * i + 2] = h[i].z;
    if (cols == 4)
      out[cols * i + 3] = h[i].w;
  }
}

// =============================================================================================
// substep stages
// =============================================================================================
// src/periodicity.hpp:25-38
template <class R>
int Sim<R>::ghostCapacity(int nReal, R band) const {
  const R sx = per_[0] ? band : R(0), sy = per_[1] ? band : R(0), sz = per_[2] ? band : R(0);
  const double ix = (dsize_[0] - R(2) * sx > R(0)) ? (double)(dsize_[0] - R(2) * sx) : 0.0;
  const double iy = (dsize_[1] - R(2) * sy > R(0)) ? (double)(dsize_[1] - R(2) * sy) : 0.0;
  const double iz = (dsize_[2] - R(2) * sz > R(0)) ? (double)(dsize_[2] - R(2) * sz) : 0.0;
  const double vt = (double)dsize_[0] * (double)dsize_[1] * (double)dsize_[2];
  if (vt <= 0.0)
    return nReal * 8;
  const double gf = (vt - ix * iy * iz) / vt;
  const double est = (gf > 0.5) ? nReal * 32.0 : nReal * gf * 4.0;
  return nReal + (int)est + 4096;
}
// src/sim.hpp:61-70
template <class R>
R Sim<R>::maxOwnedRadius() {
  if (numReal_ <= 0)
    return gs_ * baseRadius_;
  // the largest scale changes only through the scale setters, set_positions and growth: it is
  // read back once and kept until one of them runs
  if (!maxScaleValid_ || gf_ > R(0)) {
    rA_.ensure(1, false, stream_);
    rA_.zero(stream_, 1);
    ++launches_, kMaxScale<<<gridFor(numReal_), kBlock, 0, stream_>>>(d_, numReal_, rA_.p);
    KCHECK("maxScale");
    readBack(&maxScaleHost_, rA_.p, sizeof(R));
    sync();
    maxScaleValid_ = true;
  }
  return maxScaleHost_ * gs_ * baseRadius_;
}
// src/sim.hpp:119-145 (+ periodicity.hpp:43-94)
template <class R>
void Sim<R>::resetGhosts(R band) {
  ++launches_, kIota<R><<<gridFor(numReal_), kBlock, 0, stream_>>>(realIdx_.p, numReal_);
  KCHECK("iota");
  ensureCapacity(ghostCapacity(numReal_, band));
  numParticles_ = numReal_;
  if ((per_[0] || per_[1] || per_[2]) && numReal_ > 0) {
    DomainP<R> dom;
    for (int a = 0; a < 3; ++a) {
      dom.mn[a] = dmin_[a], dom.mx[a] = dmax_[a], dom.sz[a] = dsize_[a], dom.per[a] = per_[a];
    }
    iA_.ensure(numReal_ + 1, false, stream_);
    iB_.ensure(numReal_ + 1, false, stream_);
    iA_.zero(stream_, numReal_ + 1);
    ++launches_, kGhostCount<<<gridFor(numReal_), kBlock, 0, stream_>>>(d_, numReal_, dom, band, iA_.p);
    KCHECK("ghostCount");
    exclusiveSum(iA_.p, iB_.p, numReal_ + 1);
    int total = 0;
    readBack(&total, iB_.p + numReal_, sizeof(int));
    sync();
    ++launches_, kGhostWrite<<<gridFor(numReal_), kBlock, 0, stream_>>>(d_, numReal_, dom, band, iB_.p);
    KCHECK("ghostWrite");
    numParticles_ = std::min(numReal_ + total, capacity_);
  }
}
// broadphase over numParticles_ boxes of the predicted positions with margin; pairs into pairs_
// (cap entries). Returns the number of candidates, which may exceed cap (nothing written then).
template <class R>
int Sim<R>::findCollisions(R margin, int cap, int2* out, R extra) {
  const int n = numParticles_;
  const R boxCap = std::max(std::max(dsize_[0], dsize_[1]), dsize_[2]);
  if (n < 2 || numReal_ <= 0)
    return 0;
  bvhBoxes_.ensure(sizeof(Box<R>) * n, false, stream_);
  bvhNodes_.ensure(sizeof(PNode) * (2 * (size_t)n - 1), false, stream_);
  codes_.ensure(n, false, stream_);
  codesAlt_.ensure(n, false, stream_);
  bidx_.ensure(n, false, stream_);
  bidxAlt_.ensure(n, false, stream_);
  left_.ensure(n, false, stream_);
  right_.ensure(n, false, stream_);
  parent_.ensure(2 * n, false, stream_);
  flag_.ensure(n, false, stream_);
  bounds_.ensure(6, false, stream_);
  qcnt_.ensure(n, false, stream_);
  qoff_.ensure(numReal_ + 1, false, stream_);
  rowCnt_.ensure(numReal_ + 1, false, stream_);
  slots_.ensure((size_t)n * kSlots, false, stream_);
  Box<R>* prim = reinterpret_cast<Box<R>*>(bvhBoxes_.p);
  PNode* nodes = reinterpret_cast<PNode*>(bvhNodes_.p);
  BvhNodes<R> bn{prim, nullptr};
  BvhBuffers bb;
  bb.n = n;
  bb.codes = codes_.p, bb.codesAlt = codesAlt_.p, bb.idx = bidx_.p, bb.idxAlt = bidxAlt_.p;
  bb.left = left_.p, bb.right = right_.p, bb.parent = parent_.p, bb.rope = nullptr, bb.flag = flag_.p;
  bb.bounds = bounds_.p;
  bb.err = &ctr_.p->err;
  int codeBits = 63;
  if (batch_) {  // scene id leads the key: every scene is one subtree, queries stay inside it
    bvhFirst_.ensure(n, false, stream_);
    bvhLast_.ensure(n, false, stream_);
    bb.sceneOf = sceneOf_.p;
    bb.leafFirst = sceneLeafFirstD_.p;
    bb.first = bvhFirst_.p;
    bb.last = bvhLast_.p;
    codeBits = std::min(64, kSceneShift + bitsFor(numScenes_));
  }
  // The tree's topology (leaf order, links) is rebuilt when the body set changed or every
  // kBvhRebuild substeps; in between only the boxes are refitted. Any tree whose boxes contain
  // the current boxes gives the exact candidate set, so both paths give the same pairs.
  const bool rebuild = !bvhValid_ || bvhN_ != n || bvhReal_ != numReal_ || bvhAge_ >= kBvhRebuild;
  const u64 init[6] = {~0ull, ~0ull, ~0ull, 0ull, 0ull, 0ull};
  cudaCheck(cudaMemcpyAsync(bounds_.p, init, sizeof init, cudaMemcpyHostToDevice, stream_), "H2D bounds");
  ++launches_, kBoxes<<<gridFor(n), kBlock, 0, stream_>>>(d_, n, margin, boxCap, bn, bb, extra);
  KCHECK("boxes");
  if (rebuild) {
    ++launches_, kMorton<R><<<gridFor(n), kBlock, 0, stream_>>>(n, bn, bb);  // into codes_ / bidx_
    KCHECK("morton");
    // the leaf order: the broadphase's own stable radix sort of the Morton codes
    radixK_.ensure(n, false, stream_);
    radixV_.ensure(n, false, stream_);
    radixH_.ensure(256 * (size_t)radixBlocks(n), false, stream_);
    launches_ += 3 * ((codeBits + 7) / 8);
    cudaCheck(radixSortPairs(codes_.p, codesAlt_.p, bidx_.p, bidxAlt_.p, n, codeBits, radixK_.p, radixV_.p,
                             radixH_.p, stream_),
              "morton sort");
  }
  // the sorted order (this build's, or the last build's on a refit-only substep) is the sort's
  // output, in the *Alt buffers
  bb.codes = codesAlt_.p, bb.codesAlt = codes_.p, bb.idx = bidxAlt_.p, bb.idxAlt = bidx_.p;
  if (rebuild && batch_)
    ++launches_, kSceneLeafFirst<<<gridFor(numScenes_ + 1), kBlock, 0, stream_>>>(n, numScenes_, bb.codes,
                                                                                  sceneLeafFirstD_.p);
  cudaCheck(cudaMemsetAsync(flag_.p, 0, n * sizeof(int), stream_), "memset");
  cudaCheck(cudaMemsetAsync(rowCnt_.p, 0, (numReal_ + 1) * sizeof(int), stream_), "memset");
  bflag_.ensure(1, false, stream_);
  cudaCheck(cudaMemsetAsync(bflag_.p, 0, sizeof(int), stream_), "memset");
  if (rebuild) {
    ++launches_, kKarras<<<gridFor(n - 1), kBlock, 0, stream_>>>(bb);
    KCHECK("karras");
    ++launches_, kPackLeaves<R><<<gridFor(n), kBlock, 0, stream_>>>(bb, prim, nodes);
    KCHECK("leaves");
    ++launches_, kRefitPacked<<<gridFor(n), kBlock, 0, stream_>>>(bb, nodes);
    KCHECK("refit");
    ++launches_, kRopesPacked<<<gridFor(2 * n - 1), kBlock, 0, stream_>>>(bb, nodes);
    KCHECK("ropes");
    bvhValid_ = true;
    bvhN_ = n;
    bvhReal_ = numReal_;
    bvhAge_ = 0;
  } else {
    ++launches_, kRefreshLeaves<R><<<gridFor(n), kBlock, 0, stream_>>>(bb, prim, nodes);
    KCHECK("leaves");
    ++launches_, kRefitPacked<<<gridFor(n), kBlock, 0, stream_>>>(bb, nodes);
    KCHECK("refit");
  }
  ++bvhAge_;
  ++launches_, kQueryHalf<R><<<gridFor(n, 128), 128, 0, stream_>>>(bb, prim, nodes, numReal_, rowCnt_.p, qcnt_.p,
                                                                     slots_.p, bflag_.p);
  KCHECK("query");
  exclusiveSum(rowCnt_.p, qoff_.p, numReal_ + 1);
  int total = 0, err = 0, overflow = 0;
  readBack(&total, qoff_.p + numReal_, sizeof(int));
  readBack(&err, &ctr_.p->err, sizeof(int));
  readBack(&overflow, bflag_.p, sizeof(int));
  sync();
  if (err & 1)
    throw std::runtime_error("broadphase: BVH traversal exceeded its iteration bound (corrupt tree)");
  if (overflow) {
    // some query had more partners than its slots: count and write with full traversals
    cudaCheck(cudaMemsetAsync(rowCnt_.p, 0, (numReal_ + 1) * sizeof(int), stream_), "memset");
    ++launches_, kQueryFull<R, 0><<<gridFor(n, 128), 128, 0, stream_>>>(bb, prim, nodes, numReal_, rowCnt_.p,
                                                                          nullptr, nullptr, 0);
    KCHECK("query count");
    exclusiveSum(rowCnt_.p, qoff_.p, numReal_ + 1);
    readBack(&total, qoff_.p + numReal_, sizeof(int));
    readBack(&err, &ctr_.p->err, sizeof(int));
    sync();
    if (err & 1)
      throw std::runtime_error("broadphase: BVH traversal exceeded its iteration bound (corrupt tree)");
    if (total <= cap) {
      ++launches_, kQueryFull<R, 1><<<gridFor(n, 128), 128, 0, stream_>>>(bb, prim, nodes, numReal_, nullptr,
                                                                            qoff_.p, out, cap);
      KCHECK("query write");
    }
  } else if (total <= cap) {
    ++launches_, kScatterHalf<<<gridFor(n), kBlock, 0, stream_>>>(bb, qcnt_.p, slots_.p, qoff_.p, out, cap);
    KCHECK("pair scatter");
  }
  if (total <= cap) {
    ++launches_, kSortPairLists<<<gridFor(numReal_), kBlock, 0, stream_>>>(numReal_, qoff_.p, out, cap);
    KCHECK("pair sort");
  }
  return total;
}
// src/sim.hpp:82-94: grow the pair buffer and re-run when the candidates exceed it
template <class R>
int Sim<R>::findCollisionsGrow(R margin, const Q4<R>*) {
  int np = findCollisions(margin, (int)pairs_.n, pairs_.p);
  if (np > (int)pairs_.n) {
    const int grown = np + np / 2 + 64;
    pairs_.ensure(grown, false, stream_);
    maxPairs_ = grown;
    refreshDev();
    np = findCollisions(margin, (int)pairs_.n, pairs_.p);
  }
  return std::min(np, (int)pairs_.n);
}
// The step's candidate pairs through a Verlet superset (see kVerletDisplacement): the exact list,
// in canonical order, identical to findCollisionsGrow's. The superset is rebuilt (BVH query with
// every box widened by half the skin) when the body set, the margin or a scale changed, or when
// some body moved more than half the skin since the last build.
template <class R>
int Sim<R>::findCollisionsVerlet(R margin) {
  const int n = numParticles_;
  if (n < 2 || numReal_ <= 0)
    return 0;
  const R skin = R(0.5) * margin;
  const R boxCap = std::max(std::max(dsize_[0], dsize_[1]), dsize_[2]);
  // a widened box that the exact predicate would not park must not be parked either
  if (boxCap > R(0) && maxOwnedRadius() + margin + R(0.5) * skin > boxCap)
    return findCollisionsGrow(margin, posPred_.p);
  bvhBoxes_.ensure(sizeof(Box<R>) * n, false, stream_);
  bounds_.ensure(6, false, stream_);
  rA_.ensure(1, false, stream_);
  Box<R>* prim = reinterpret_cast<Box<R>*>(bvhBoxes_.p);
  BvhNodes<R> bn{prim, nullptr};
  BvhBuffers bb;
  bb.n = n;
  bb.bounds = bounds_.p;
  bb.err = &ctr_.p->err;
  const bool fresh = vValid_ && vN_ == n && vReal_ == numReal_ && vMargin_ == margin;
  for (int attempt = 0; attempt < 2; ++attempt) {
    const bool useOld = fresh && attempt == 0;
    if (!useOld) {
      // (re)build the superset: BVH query with the widened boxes, into vpairs_ (grown on demand)
      int nv = findCollisions(margin, (int)vpairs_.n, vpairs_.p, R(0.5) * skin);
      if (nv > (int)vpairs_.n) {
        vpairs_.ensure((size_t)nv + nv / 2 + 64, false, stream_);
        nv = findCollisions(margin, (int)vpairs_.n, vpairs_.p, R(0.5) * skin);
      }
      vCount_ = nv;
      vRef_.ensure(n, false, stream_);
      vRefReal_.ensure(n, false, stream_);
      cudaCheck(cudaMemcpyAsync(vRef_.p, posPred_.p, n * sizeof(Q4<R>), cudaMemcpyDeviceToDevice, stream_), "D2D");
      cudaCheck(cudaMemcpyAsync(vRefReal_.p, realIdx_.p, n * sizeof(int), cudaMemcpyDeviceToDevice, stream_), "D2D");
      vValid_ = true, vN_ = n, vReal_ = numReal_, vMargin_ = margin;
    }
    // exact boxes of this substep, displacement since the build, and the filter
    const u64 init[6] = {~0ull, ~0ull, ~0ull, 0ull, 0ull, 0ull};
    cudaCheck(cudaMemcpyAsync(bounds_.p, init, sizeof init, cudaMemcpyHostToDevice, stream_), "H2D bounds");
    ++launches_, kBoxes<<<gridFor(n), kBlock, 0, stream_>>>(d_, n, margin, boxCap, bn, bb);
    rA_.zero(stream_, 1);
    ++launches_, kVerletDisplacement<<<gridFor(n), kBlock, 0, stream_>>>(d_, n, vRef_.p, vRefReal_.p, rA_.p);
    const int nc = vCount_;
    vKeep_.ensure((size_t)nc + 1, false, stream_);
    vOff_.ensure((size_t)nc + 1, false, stream_);
    if (nc > 0)
      ++launches_, kFilterPairs<<<gridFor(nc), kBlock, 0, stream_>>>(vpairs_.p, nc, prim, vKeep_.p);
    cudaCheck(cudaMemsetAsync(vKeep_.p + nc, 0, sizeof(int), stream_), "memset");
    exclusiveSum(vKeep_.p, vOff_.p, nc + 1);
    KCHECK("verlet filter");
    int total = 0;
    R disp = 0;
    readBack(&total, vOff_.p + nc, sizeof(int));
    readBack(&disp, rA_.p, sizeof(R));
    sync();
    if (useOld && !(disp <= R(0.5) * skin))
      continue;  // some body left its widened box: rebuild and filter again
    if (total > (int)pairs_.n) {
      pairs_.ensure((size_t)total + total / 2 + 64, false, stream_);
      maxPairs_ = (int)pairs_.n;
      refreshDev();
    }
    if (nc > 0)
      ++launches_, kCompactPairs<<<gridFor(nc), kBlock, 0, stream_>>>(vpairs_.p, nc, vKeep_.p, vOff_.p, pairs_.p,
                                                                      (int)pairs_.n);
    KCHECK("verlet compact");
    return total;
  }
  throw std::runtime_error("broadphase: a freshly built candidate superset failed its own displacement check");
}
template <class R>
void Sim<R>::detectAll(R margin) {
  const int np = verlet_ ? findCollisionsVerlet(margin) : findCollisionsGrow(margin, posPred_.p);
  mark(ST_NARROW);
  ++launches_, kResetCounters<<<1, 1, 0, stream_>>>(ctr_.p);
  NarrowP<R> P{margin, gs_, (int)planesHost_.size(), (int)wallsHost_.size(), pairMatHost_.empty() ? 0 : 1};
  const bool shell = shape_.numPoints > 0;
  const int nr = numReal_;
  iA_.ensure(std::max(np, 1) + 1, false, stream_);
  iB_.ensure(std::max(np, 1) + 1, false, stream_);
  iC_.ensure(nr + 1, false, stream_);
  iD_.ensure(nr + 1, false, stream_);
  iE_.ensure(2 * (size_t)nr + 2, false, stream_);
  iA_.zero(stream_, np + 1);
  iC_.zero(stream_, nr + 1);
  iD_.zero(stream_, nr + 1);
  int* cntW = iE_.p;
  int* offP = iE_.p + (nr + 1);
  // counts
  if (np > 0) {
    if (shell)
      ++launches_, kNarrowShell<R, 0><<<gridFor((long)np * 32), kBlock, shellStageBytes(), stream_>>>(
          d_, np, P, iA_.p, nullptr, shellStageBytes());
    else
      ++launches_, kNarrowSphere<R, 0><<<gridFor(np), kBlock, 0, stream_>>>(d_, np, P, iA_.p, nullptr);
    KCHECK("narrow count");
  }
  const bool boundary = nr > 0 && (P.numPlanes > 0 || P.numWalls > 0);
  if (boundary) {
    if (shell)
      ++launches_, kBoundary<R, 0><<<gridFor((long)nr * 32), kBlock, 0, stream_>>>(d_, nr, P, iC_.p, iD_.p, nullptr, nullptr, 0, 0);
    else
      ++launches_, kBoundarySphere<R, 0><<<gridFor(nr), kBlock, 0, stream_>>>(d_, nr, P, iC_.p, iD_.p, nullptr, 0);
    KCHECK("boundary count");
  }
  exclusiveSum(iA_.p, iB_.p, np + 1);
  exclusiveSum(iC_.p, offP, nr + 1);
  exclusiveSum(iD_.p, cntW, nr + 1);
  // one read-back: the three totals and the counters the count passes updated (max overlap, errors)
  int tot[3] = {0, 0, 0};
  Counters<R> c;
  readBack(&tot[0], iB_.p + np, sizeof(int));
  readBack(&tot[1], offP + nr, sizeof(int));
  readBack(&tot[2], cntW + nr, sizeof(int));
  readBack(&c, ctr_.p, sizeof c);
  sync();
  if (c.err & kErrBarrier) {
    clearLoopError();
    throw CudaError("a grid-wide barrier of a persistent loop timed out (blocks not co-resident)");
  }
  if (np > 0 && tot[0] > 0) {
    if (shell)
      ++launches_, kNarrowShell<R, 1><<<gridFor((long)np * 32), kBlock, shellStageBytes(), stream_>>>(
          d_, np, P, nullptr, iB_.p, shellStageBytes());
    else {
      // iA_ (the 0/1 counts) is free after the scan: it receives the hit pair of every slot
      ++launches_, kHitIndex<<<gridFor(np), kBlock, 0, stream_>>>(np, iB_.p, iA_.p);
      ++launches_, kNarrowSphereWrite<R><<<gridFor(tot[0]), kBlock, 0, stream_>>>(d_, tot[0], P, iA_.p);
    }
    KCHECK("narrow write");
  }
  if (boundary && tot[1] + tot[2] > 0 && tot[0] < maxContacts_) {
    if (shell)
      ++launches_, kBoundary<R, 1><<<gridFor((long)nr * 32), kBlock, 0, stream_>>>(d_, nr, P, nullptr, nullptr, offP, cntW,
                                                                                 tot[0], tot[0] + tot[1]);
    else {
      if (tot[1] > 0)
        ++launches_, kBoundarySphere<R, 1><<<gridFor(nr), kBlock, 0, stream_>>>(d_, nr, P, nullptr, nullptr, offP, tot[0]);
      if (tot[2] > 0)
        ++launches_, kBoundaryWallSphere<R><<<gridFor(tot[2]), kBlock, 0, stream_>>>(d_, tot[2], nr, P, cntW,
                                                                                    tot[0] + tot[1]);
    }
    KCHECK("boundary write");
  }
  const long total = (long)tot[0] + tot[1] + tot[2];
  lastTot_[0] = tot[0], lastTot_[1] = tot[1], lastTot_[2] = tot[2];
  if (batch_ && total > maxContacts_)
    throw std::runtime_error("batched scenes: the contact buffer overflowed (raise the capacity)");
  // the write passes leave the counters unchanged: the snapshot above is current
  c.pairCount = np;
  c.contactTotal = (int)std::min<long>(total, 0x7fffffff);
  c.contactCount = (int)std::min<long>(total, maxContacts_);
  detectCounters_ = c;
  cudaCheck(cudaMemcpyAsync(ctr_.p, &detectCounters_, sizeof(Counters<R>), cudaMemcpyHostToDevice, stream_),
            "H2D counters");
  // topology reuse: does this contact list equal the previous one? (recorded for the next substep)
  const int ncs = c.contactCount;
  topoFlags_.ensure(2, false, stream_);
  const int differ0 = (ncs != prevNc_ || numParticles_ != prevNb_) ? 1 : 0;
  cudaCheck(cudaMemsetAsync(topoFlags_.p, 0, 2 * sizeof(int), stream_), "memset");
  if (differ0)
    cudaCheck(cudaMemcpyAsync(topoFlags_.p, &kOne, sizeof(int), cudaMemcpyHostToDevice, stream_), "H2D");
  if (ncs > 0) {
    prevCab_.ensure(ncs, true, stream_);
    ++launches_, kSameInt2<<<gridFor(ncs), kBlock, 0, stream_>>>(cab_.p, prevCab_.p, ncs, topoFlags_.p);
    KCHECK("same contacts");
  }
  prevNc_ = ncs;
  prevNb_ = numParticles_;
}

// src/contact_preprocessing.hpp:378-471
template <class R>
int Sim<R>::reduceManifolds(int nc) {
  if (nc <= 0)
    return 0;
  const int kb = bitsFor((long)numParticles_ + 1);
  // the grouping (sorted keys, permutation, segments, manifold count) depends on the contact
  // list's body pairs only: unchanged list -> keep it. The check costs a read-back, so it is made
  // after a substep whose list was unchanged, and every 4th substep otherwise.
  if (topoValid_ && nc == prevNcM_ && (lastSame_ || (topoChecks_++ & 3) == 0)) {
    int differ = 1;
    readBack(&differ, topoFlags_.p, sizeof(int));
    sync();
    lastSame_ = differ == 0;
    if (lastSame_) {
      ++reuse_[0];
      const int nm = prevNm_;
      ++launches_, kReduceManifolds<<<gridFor(nm), kBlock, 0, stream_>>>(d_, nm, nc, kb, segStart_.p, ckeysS_.p,
                                                                          cperm_.p);
      KCHECK("reduce manifolds");
      return nm;
    }
  } else {
    lastSame_ = false;
  }
  ckeys_.ensure(nc, false, stream_);
  ckeysS_.ensure(nc, false, stream_);
  cpermIn_.ensure(nc, false, stream_);
  cperm_.ensure(nc, false, stream_);
  head_.ensure(nc, false, stream_);
  headScan_.ensure(nc, false, stream_);
  segStart_.ensure(nc + 1, false, stream_);
  // the narrowphase's list is in key order up to its boundary contacts: the stable sort is a rank
  // scatter (kContactRanks), checked on the device; a list it rejects is sorted after all
  static const bool forceSort = std::getenv("PDEM_CONTACT_SORT") != nullptr;
  const bool ranked = !forceSort && numReal_ > 0 && (long)lastTot_[0] + lastTot_[1] + lastTot_[2] == nc;
  int hostBad[2] = {0, 0};  // [0] manifold count, [1] the rank scatter's rejection
  auto groups = [&](bool sortNow) {
    if (sortNow) {
      ++launches_, kContactKeys<R><<<gridFor(nc), kBlock, 0, stream_>>>(d_, nc, kb, ckeys_.p, cpermIn_.p);
      KCHECK("contact keys");
      sortPairs(ckeys_.p, ckeysS_.p, cpermIn_.p, cperm_.p, nc, 2 * kb);
    } else {
      const int nr = numReal_;
      rankBad_.ensure(1, false, stream_);
      rankBad_.zero(stream_, 1);
      ++launches_, kContactRanks<R><<<gridFor(nc), kBlock, 0, stream_>>>(d_, nc, lastTot_[0], lastTot_[1], nr,
                                                                         iE_.p + (nr + 1), iE_.p, kb, ckeysS_.p,
                                                                         cperm_.p, rankBad_.p);
      KCHECK("contact ranks");
    }
    ++launches_, kSegHeads<<<gridFor(nc), kBlock, 0, stream_>>>(nc, ckeysS_.p, head_.p);
    KCHECK("seg heads");
    inclusiveSum(head_.p, headScan_.p, nc);
    readBack(&hostBad[0], headScan_.p + nc - 1, sizeof(int));
    if (!sortNow)
      readBack(&hostBad[1], rankBad_.p, sizeof(int));
    sync();
  };
  groups(!ranked);
  if (ranked && hostBad[1]) {
    ++rankStats_[1];
    hostBad[1] = 0;
    groups(true);
  } else if (ranked) {
    ++rankStats_[0];
  }
  const int nm = hostBad[0];
  ++launches_, kSegStarts<<<gridFor(nc), kBlock, 0, stream_>>>(nc, headScan_.p, segStart_.p);
  KCHECK("seg starts");
  ++launches_, kReduceManifolds<<<gridFor(nm), kBlock, 0, stream_>>>(d_, nm, nc, kb, segStart_.p, ckeysS_.p, cperm_.p);
  KCHECK("reduce manifolds");
  prevNm_ = nm;
  prevNcM_ = nc;
  return nm;
}

// Both Jones-Plassmann colourings of the substep in one cooperative launch
// (src/solver_velocity.hpp:277-374 for the manifolds, src/solver_position.hpp:155-241 for the
// contacts); one read-back gives each graph's colour count and uncoloured entries.
template <class R>
void Sim<R>::colorBoth(int nm, int nc, int& ncolV, int& velLeft, int& ncolP, int& posLeft) {
  ncolV = ncolP = velLeft = posLeft = 0;
  const int nbM = numReal_, nbC = numParticles_;
  const int neM = (nm > 0 && nbM > 0) ? nm : 0, neC = (nc > 0 && nbC > 0) ? nc : 0;
  if (neM == 0 && neC == 0)
    return;
  mask_.ensure(std::max(nbM, 1), false, stream_);
  maskP_.ensure(std::max(nbC, 1), false, stream_);
  winner_.ensure(std::max(nbM, 1), false, stream_);
  winner2_.ensure(std::max(nbM, 1), false, stream_);
  winnerP_.ensure(std::max(nbC, 1), false, stream_);
  winnerP2_.ensure(std::max(nbC, 1), false, stream_);
  colorAux_.ensure(12, false, stream_);
  colorListM_.ensure(2 * std::max(neM, 1), false, stream_);
  colorListC_.ensure(2 * std::max(neC, 1), false, stream_);
  // per job: the blocks' list lengths (up to 4 blocks per SM), then the tail's two lists
  const int maxGrid = 4 * numSMs_;
  colorTail_.ensure(2 * (maxGrid + 2 * (size_t)kColorTailMax), false, stream_);
  int* tm = colorTail_.p;
  int* tc = colorTail_.p + maxGrid + 2 * kColorTailMax;
  ColorJob jm{neM, nbM, mColor_.p, winner_.p, winner2_.p, mask_.p, colorAux_.p, colorListM_.p,
              colorListM_.p + std::max(neM, 1), tm, tm + maxGrid, tm + maxGrid + kColorTailMax, std::min(colorTailAt_, kColorTailMax)};
  ColorJob jc{neC, nbC, cColor_.p, winnerP_.p, winnerP2_.p, maskP_.p, colorAux_.p + 6, colorListC_.p,
              colorListC_.p + std::max(neC, 1), tc, tc + maxGrid, tc + maxGrid + kColorTailMax, std::min(colorTailAt_, kColorTailMax)};
  if (!batch_) {  // the colour orders come out of the same launch (the batched form orders by scene)
    colorHist_.ensure(2 * 64 * (size_t)maxGrid, false, stream_);
    if (neM > 0) {
      mOrder_.ensure(neM, false, stream_);
      mOff_.ensure(66, false, stream_);
      jm.order = mOrder_.p, jm.off = mOff_.p, jm.hist = colorHist_.p;
    }
    if (neC > 0) {
      cOrder_.ensure(neC, false, stream_);
      cOff_.ensure(66, false, stream_);
      jc.order = cOrder_.p, jc.off = cOff_.p, jc.hist = colorHist_.p + 64 * maxGrid;
    }
  }
  gbar_.ensure(2, false, stream_);
  const GridBar gb{gbar_.p, &ctr_.p->err, barrierSleepNs_, barrierSpins_};
  // the tail in shared memory when the hand-over fits its tables
  const bool tailShared = std::min(colorTailAt_, kColorTailMax) <= kTailShEntries;
  jm.tailShared = jc.tailShared = tailShared ? 1 : 0;
  const size_t tailSmem = tailShared ? sizeof(TailShared) : 0;
  const bool inCluster =
      std::max(neM, neC) <= colorClusterEntries_ && colorBlock_ == kColorBlock &&
      (cudaMemsetAsync(gbar_.p, 0, 2 * sizeof(unsigned), stream_) == cudaSuccess) &&
      launchClusterCfg(kColorBoth<R, true>, sweepClusterBlocks_, kColorBlock, tailSmem, d_, jm, jc,
                       std::max(nbM, nbC) + 2, gb, (const int*)topoFlags_.p, topoValid_ ? 1 : 0);
  // batched form: the launch-shape autotuner's colouring candidates (see colorTuning_)
  const bool tuneColor = !inCluster && batch_ && colorTuning_;
  const int slot = colorTuneStep_ % (kColorTuneCands * kTuneRounds);
  if (tuneColor) {
    if (!colorTuneEv_[0][0])
      for (auto& pr : colorTuneEv_)
        for (auto& e : pr)
          cudaCheck(cudaEventCreate(&e), "event");
    colorBlock_ = kColorTuneBlocks[colorTuneStep_ % kColorTuneCands];
    cudaCheck(cudaEventRecord(colorTuneEv_[slot][0], stream_), "event");
  }
  if (!inCluster)
    launchCoopSmem(kColorBoth<R>, colorBlock_, tailSmem, d_, jm, jc, std::max(nbM, nbC) + 2, gb,
                   (const int*)topoFlags_.p, topoValid_ ? 1 : 0);
  if (tuneColor) {
    cudaCheck(cudaEventRecord(colorTuneEv_[slot][1], stream_), "event");
    if (++colorTuneStep_ == kColorTuneCands * kTuneRounds) {
      sync();
      float best = 0;
      for (int c = 0; c < kColorTuneCands; ++c) {
        float tot = 0;
        for (int r = 0; r < kTuneRounds; ++r) {
          float ms = 0;
          cudaCheck(cudaEventElapsedTime(&ms, colorTuneEv_[r * kColorTuneCands + c][0],
                                         colorTuneEv_[r * kColorTuneCands + c][1]), "event");
          tot += ms;
        }
        colorTuneMs_[c] = tot / kTuneRounds;
        if (c == 0 || tot < best) {
          best = tot;
          colorBlock_ = kColorTuneBlocks[c];
        }
      }
      colorTuning_ = false;
    }
  }
  KCHECK("colour loop");
  int res[12], err = 0, differ[2] = {1, 1};
  readBack(res, colorAux_.p, sizeof res);
  readBack(&err, &ctr_.p->err, sizeof err);
  readBack(differ, topoFlags_.p, sizeof differ);
  sync();
  keptC_ = topoValid_ && differ[0] == 0;
  keptM_ = topoValid_ && differ[1] == 0;
  reuse_[1] += keptC_ ? 1 : 0;
  reuse_[2] += keptM_ ? 1 : 0;
  if (err & kErrBarrier) {
    clearLoopError();
    throw CudaError("colouring: a grid-wide barrier timed out");
  }
  if (neM > 0) {
    ncolV = res[3] + 1;
    velLeft = res[4];
    colorRounds_[0] = res[5];
  }
  if (neC > 0) {
    ncolP = res[9] + 1;
    posLeft = res[10];
    colorRounds_[1] = res[11];
  }
}
// batched form: the (scene, colour) execution order, scene s's colour c occupying
// [off[s * 64 + c], off[s * 64 + c + 1]) (the single-scene orders come out of kColorBoth)
template <class R>
void Sim<R>::colorOrder(bool manifold, int ne, int ncol) {
  (void)ncol;
  DBuf<int>& order = manifold ? mOrder_ : cOrder_;
  DBuf<int>& off = manifold ? mOff_ : cOff_;
  order.ensure(ne, false, stream_);
  off.ensure((size_t)numScenes_ * 64 + 2, false, stream_);
  // one block per scene over its slice of the body-sorted ranges (batchBounds' first entries)
  ++launches_, kColorOrderScenes<<<numScenes_, 256, 0, stream_>>>(manifold ? mColor_.p : cColor_.p,
                                                                 manifold ? sceneManFirstD_.p : sceneConFirstD_.p,
                                                                 manifold ? 1 : 3, numScenes_, ne, order.p, off.p);
  KCHECK("color order (scenes)");
}
// per-body incidence lists in ascending source order. kind 0: manifolds x real bodies,
// 1: contacts x real bodies, 2: contacts x raw body slots
template <class R>
void Sim<R>::buildIncidence(int kind, int ne, int nb) {
  incKind_ = kind;
  incNe_ = ne;
  const int n2 = 2 * ne;
  incKeys_.ensure(std::max(n2, 1), false, stream_);
  incKeysS_.ensure(std::max(n2, 1), false, stream_);
  incVals_.ensure(std::max(n2, 1), false, stream_);
  incValsS_.ensure(std::max(n2, 1), false, stream_);
  incOff_.ensure(nb + 2, false, stream_);
  if (ne <= 0) {
    incOff_.zero(stream_, nb + 1);
    return;
  }
  if (kind == 0)
    ++launches_, kIncidenceKeys<R, 0><<<gridFor(ne), kBlock, 0, stream_>>>(d_, ne, incKeys_.p, incVals_.p, nb);
  else if (kind == 1)
    ++launches_, kIncidenceKeys<R, 1><<<gridFor(ne), kBlock, 0, stream_>>>(d_, ne, incKeys_.p, incVals_.p, nb);
  else if (kind == 2)
    ++launches_, kIncidenceKeys<R, 2><<<gridFor(ne), kBlock, 0, stream_>>>(d_, ne, incKeys_.p, incVals_.p, nb);
  else
    ++launches_, kIncidenceKeys<R, 3><<<gridFor(ne), kBlock, 0, stream_>>>(d_, ne, incKeys_.p, incVals_.p, nb);
  KCHECK("incidence keys");
  sortPairs(incKeys_.p, incKeysS_.p, incVals_.p, incValsS_.p, n2, bitsFor(nb));
  ++launches_, kLowerBoundOffsets<int><<<gridFor(nb + 1), kBlock, 0, stream_>>>(n2, incKeysS_.p, nb, incOff_.p);
  KCHECK("incidence offsets");
}

// =============================================================================================
// the substep: src/sim.hpp:97-488
// =============================================================================================
template <class R>
void Sim<R>::step(R dt) {
  dt_ = dt;
  demStep();
}

template <class R>
void Sim<R>::demStep() {
  const int B = kBlock;
  cudaStream_t s = stream_;
  ++substepId_;
  mark(ST_PREDICT);
  if (batch_)
    batchBegin();
  if (gf_ != R(-1) && gr_ != R(0)) {
    gf_ *= std::exp(gr_ * dt_);
    if (gf_ > R(1))
      gf_ = R(1);
  }
  if (gf_ > R(0) && numReal_ > 0) {
    vValid_ = false;  // the radii change this substep
    ++launches_, kGrowthScales<<<gridFor(numReal_), B, 0, s>>>(d_, numReal_, gf_);
    KCHECK("growth");
  }
  const R maxRad = maxOwnedRadius();
  const R margin = R(0.1) * maxRad;
  const V3<R> g{g_[0], g_[1], g_[2]};
  if (numReal_ > 0) {
    ++launches_, kPredict<<<gridFor(numReal_), B, 0, s>>>(d_, numReal_, g, dt_);
    KCHECK("predict");
  }
  mark(ST_GHOSTS);
  resetGhosts(maxRad);
  if (numParticles_ > 0) {
    ++launches_, kRadii<<<gridFor(numParticles_), B, 0, s>>>(d_, numParticles_, gs_, baseRadius_);
    KCHECK("radii");
  }
  mark(ST_BROAD);
  detectAll(margin);
  Counters<R> c0 = detectCounters_;  // the device counters as detectAll left them
  const int nc = c0.contactCount;
  mark(ST_MANIFOLD);
  const int nm = reduceManifolds(nc);
  if (batch_)
    batchBounds(nm);
  // topology reuse, manifold side: real ends and activity of every manifold vs the previous substep
  if (nm != prevNmSig_)
    cudaCheck(cudaMemcpyAsync(topoFlags_.p + 1, &kOne, sizeof(int), cudaMemcpyHostToDevice, s), "H2D");
  if (nm > 0) {
    prevMsig_.ensure(nm, true, s);
    ++launches_, kSameManifolds<<<gridFor(nm), B, 0, s>>>(d_, nm, prevMsig_.p, topoFlags_.p + 1);
    KCHECK("same manifolds");
  }
  prevNmSig_ = nm;
  c0.manifoldCount = nm;
  c0.velDone = c0.stabRun = c0.stabDone = c0.posDone = 0;
  cudaCheck(cudaMemcpyAsync(ctr_.p, &c0, sizeof c0, cudaMemcpyHostToDevice, s), "H2D counters");

  const bool friction = (mu_ > R(0) || wallFrictionMax_ > R(0));
  const bool gNZ = (g_[0] != R(0) || g_[1] != R(0) || g_[2] != R(0));
  const bool legacyFriction = friction && !(gNZ && useGS_);
  if (batch_ && legacyFriction)
    throw std::runtime_error("batched scenes: the Jacobi friction path (zero gravity) is not supported");
  if (legacyFriction) {
    planeFric_.zero(s);
    if (nc > 0)
      ++launches_, kPlaneLoad<<<gridFor(nc), B, 0, s>>>(d_, nc);
    KCHECK("plane load");
  }
  mark(ST_COLOR_V);
  // both colourings now: the contact graph is fixed since the narrowphase
  int velLeft = 0, posLeft = 0, ncolV = 0, ncolP = 0;
  keptM_ = keptC_ = false;
  if (useGS_)
    colorBoth(nm, nc, ncolV, velLeft, ncolP, posLeft);
  ncolVLast_ = ncolV, ncolPLast_ = ncolP;
  if (batch_ && (velLeft > 0 || posLeft > 0))
    throw std::runtime_error("batched scenes: uncoloured entries (Jacobi fallback) are not supported");
  // an unchanged graph keeps its colours, hence its colour order
  if (batch_ && useGS_ && ncolV > 0 && !keptM_)
    colorOrder(true, nm, ncolV);
  if (batch_ && useGS_ && ncolP > 0 && !keptC_)
    colorOrder(false, nc, ncolP);
  const bool usePGS = gNZ && useGS_;
  const R gMag = std::sqrt(g_[0] * g_[0] + g_[1] * g_[1] + g_[2] * g_[2]);
  const V3<R> gHat = gNZ ? V3<R>{g_[0] / gMag, g_[1] / gMag, g_[2] / gMag} : V3<R>{0, 0, 0};
  const bool needInc = (usePGS && nm > 0) || ((velLeft > 0 || !useGS_) && nm > 0);
  if (needInc && !(keptM_ && incKind_ == 0 && incNe_ == nm))
    buildIncidence(0, nm, numReal_);
  Incidence incM{incOff_.p, incValsS_.p};
  mark(ST_WARM);
  if (usePGS && nm > 0) {
    ++launches_, kGatherWarm<<<gridFor(nm), B, 0, s>>>(d_, nm, prevPairCount_);
    KCHECK("gather warm");
    logSupportGraph(nm, gHat);
    sideFlags_.zero(s, nm);
    ++launches_, kVn0<<<gridFor(nm), B, 0, s>>>(d_, nm, gr_);
    ++launches_, kWarmApply<<<gridFor(numReal_), B, 0, s>>>(d_, numReal_, incM);
    ++launches_, kWarmProject<<<gridFor(nm), B, 0, s>>>(d_, nm);
    KCHECK("warm start");
  } else if (usePGS) {
    logSupportGraph(0, gHat);  // no manifolds: the levels still decay this substep
  }
  mark(ST_VELOCITY);
  SolveP<R> sp{gr_, eN_, eT_, mu_, R(0), dt_, ncolV};
  const R vRest = R(2) * dt_ * std::sqrt(g_[0] * g_[0] + g_[1] * g_[1] + g_[2] * g_[2]);
  sp.vRest = vRest;
  // Jacobi scratch
  if (nm > 0 && (velLeft > 0 || !useGS_)) {
    rA_.ensure(nm, false, s);
    iC_.ensure(nm, false, s);
  }
  // the whole loop as one persistent launch when every sweep is colours only
  const bool velPersistent = useGS_ && !legacyFriction && velLeft == 0 && ncolV > 0 && velIters_ > 0;
  if (velPersistent) {
    gbar_.ensure(2, false, s);
    const GridBar gb{gbar_.p, &ctr_.p->err, barrierSleepNs_, barrierSpins_};
    const R thr = usePGS ? R(0.02) * vRest : vRest;
    ctl(CTL_VEL_BEGIN, R(0), 0);
    if (batch_)
      tuneBegin();
    if (batch_ && usePGS)
      ++launches_, kSweepScenes<R, 0, 1><<<numScenes_, sceneBlock(), 0, s>>>(d_, sceneLpt_.p, mOrder_.p, mOff_.p, velIters_, sp, thr);
    else if (batch_)
      ++launches_, kSweepScenes<R, 1, 1><<<numScenes_, sceneBlock(), 0, s>>>(d_, sceneLpt_.p, mOrder_.p, mOff_.p, velIters_, sp, thr);
    else if (usePGS && !(nm <= sweepClusterEntries_ &&
                         launchCluster(kSweepLoop<R, 3, 1, true>, d_, (const int*)mOrder_.p, (const int*)mOff_.p,
                                       ncolV, velIters_, sp, thr, gb, packPgs(nm, ncolV))))
      launchCoop(kSweepLoop<R, 0, 1>, d_, (const int*)mOrder_.p, (const int*)mOff_.p, ncolV, velIters_, sp, thr, gb,
                 PgsRecs<R>{});
    else if (!usePGS && !(nm <= sweepClusterEntries_ &&
                          launchCluster(kSweepLoop<R, 1, 1, true>, d_, (const int*)mOrder_.p, (const int*)mOff_.p,
                                        ncolV, velIters_, sp, thr, gb, PgsRecs<R>{})))
      launchCoop(kSweepLoop<R, 1, 1>, d_, (const int*)mOrder_.p, (const int*)mOff_.p, ncolV, velIters_, sp, thr, gb,
                 PgsRecs<R>{});
    KCHECK("velocity loop");
  }
  // no colours and no fallback: the first sweep is empty, its END finds maxApproach = 0 <= thr
  // and the loop is done, so one BEGIN/END pair stands for the whole loop
  const bool velEmpty = useGS_ && !legacyFriction && velLeft == 0 && ncolV <= 0 && velIters_ > 0;
  if (velEmpty) {
    ctl(CTL_VEL_BEGIN, R(0), 0);
    ctl(CTL_VEL_END, usePGS ? R(0.02) * vRest : vRest, 0);
  }
  for (int it = 0; it < (velPersistent || velEmpty ? 0 : velIters_); ++it) {
    if (legacyFriction && nc > 0) {
      // runs at the top of every iteration the loop reaches (src/sim.hpp:224-226): with the
      // coloured solve the adaptive stop ends the loop, so it is gated on the loop flag
      ++launches_, kAccumNormal<<<gridFor(nc), B, 0, s>>>(d_, nc, gr_, useGS_ ? 1 : 0);
      KCHECK("accum normal");
    }
    if (useGS_) {
      ctl(CTL_VEL_BEGIN, R(0), 0);
      for (int col = 0; col < ncolV; ++col) {
        if (usePGS)
          ++launches_, kPGSColor<<<gridFor(nm), B, 0, s>>>(d_, mOrder_.p, mOff_.p, col, sp, 1);
        else
          ++launches_, kGSColor<<<gridFor(nm), B, 0, s>>>(d_, mOrder_.p, mOff_.p, col, sp, 1);
      }
      KCHECK("velocity sweep");
      if (velLeft > 0) {
        ++launches_, kJacobiImpulses<<<gridFor(nm), B, 0, s>>>(d_, nm, sp, 1, rA_.p, iC_.p, 1);
        ++launches_, kJacobiGather<<<gridFor(numReal_), B, 0, s>>>(d_, numReal_, incM, rA_.p, iC_.p, 1);
        ++launches_, kApplyVelAveraged<<<gridFor(numParticles_), B, 0, s>>>(d_, numParticles_, 1);
        KCHECK("velocity jacobi fallback");
      }
      ctl(CTL_VEL_END, usePGS ? R(0.02) * vRest : vRest, 0);
    } else {
      if (nm > 0) {
        ++launches_, kJacobiImpulses<<<gridFor(nm), B, 0, s>>>(d_, nm, sp, 0, rA_.p, iC_.p, 0);
        ++launches_, kJacobiGather<<<gridFor(numReal_), B, 0, s>>>(d_, numReal_, incM, rA_.p, iC_.p, 0);
      }
      ++launches_, kApplyVelAveraged<<<gridFor(numParticles_), B, 0, s>>>(d_, numParticles_, 0);
      KCHECK("velocity jacobi");
    }
  }
  mark(ST_STAB);
  if (usePGS) {
    const R vRestS = R(2) * dt_ * gMag;
    if (stabMode_ == 4 && batch_)
      throw std::runtime_error("batched scenes: stabilization mode 'ordered' is not supported");
    if (stabMode_ == 2 && batch_)
      throw std::runtime_error("batched scenes: stabilization mode 'multilevel' is not supported");
    ctl(CTL_STAB_DECIDE, vRestS, stabMode_);
    // periodic scenes: split the manifolds for the ledger order now, so the number of ghost
    // manifolds (the host sizes their sort with it) comes back with the decision below
    ledgerSplit_ = nm > 0 && !keptM_ && numParticles_ != numReal_ && (stabMode_ == 1 || stabMode_ == 3 || stabMode_ == 4);
    if (ledgerSplit_) {
      const int kbL = bitsFor((long)numParticles_ + 1);
      lkeysIn_.ensure(nm, false, s);
      ledFlag_.ensure((size_t)nm + 1, false, s);
      ledPos_.ensure((size_t)nm + 1, false, s);
      ledGhost_.ensure((size_t)nm + 1, false, s);
      ledGPos_.ensure((size_t)nm + 1, false, s);
      ++launches_, kLedgerClass<R><<<gridFor(nm), B, 0, s>>>(d_, nm, kbL, numReal_, pairKeys_.p, lkeysIn_.p, ledFlag_.p,
                                                             ledGhost_.p);
      cudaCheck(cudaMemsetAsync(ledFlag_.p + nm, 0, sizeof(int), s), "memset");
      cudaCheck(cudaMemsetAsync(ledGhost_.p + nm, 0, sizeof(int), s), "memset");
      exclusiveSum(ledFlag_.p, ledPos_.p, nm + 1);
      exclusiveSum(ledGhost_.p, ledGPos_.p, nm + 1);
      KCHECK("ledger split");
      readBack(&ledgerGhosts_, ledGPos_.p + nm, sizeof(int));
    }
    // the pass runs only when the main sweeps left a residual (src/sim.hpp:282): read the
    // decision so an untriggered pass costs nothing
    const bool stabRun = stabMode_ != 0 && readCounters().stabRun;
    if (stabRun && stabMode_ == 4) {
      SolveP<R> ss = sp;
      ss.vRest = vRestS;
      orderedStabilization(nm, gHat, ss, vRestS);
    } else if (stabRun && stabMode_ == 2) {
      SolveP<R> ss = sp;
      ss.vRest = vRestS;
      multilevelStabilization(nm, ncolV, ss, vRestS, gMag);
    } else if (stabRun) {
      if (stabMode_ == 1 && nm > 0) {
        ensureGrounded();
        ++launches_, kSideFlags<<<gridFor(nm), B, 0, s>>>(d_, nm, gHat, R(8) * dt_ * gMag, R(8) * dt_ * gMag);
      }
      SolveP<R> ss = sp;
      ss.vRest = vRestS;
      const int iters = stabMode_ == 1 ? 2 * velIters_ : 256;
      const bool stabPersistent = ncolV > 0;
      if (stabPersistent) {
        gbar_.ensure(2, false, s);
        const GridBar gb{gbar_.p, &ctr_.p->err, barrierSleepNs_, barrierSpins_};
        ctl(CTL_STAB_BEGIN, R(0), 0);
        if (batch_)
          ++launches_, kSweepScenes<R, 0, 2><<<numScenes_, sceneBlock(), 0, s>>>(d_, sceneLpt_.p, mOrder_.p, mOff_.p, iters, ss, vRestS);
        else if (!(nm <= sweepClusterEntries_ &&
                   launchCluster(kSweepLoop<R, 3, 2, true>, d_, (const int*)mOrder_.p, (const int*)mOff_.p, ncolV,
                                 iters, ss, vRestS, gb, packPgs(nm, ncolV))))
          launchCoop(kSweepLoop<R, 0, 2>, d_, (const int*)mOrder_.p, (const int*)mOff_.p, ncolV, iters, ss, vRestS, gb,
                     PgsRecs<R>{});
      }
      for (int it = 0; it < (stabPersistent ? 0 : iters); ++it) {
        ctl(CTL_STAB_BEGIN, R(0), 0);
        for (int col = 0; col < ncolV; ++col)
          ++launches_, kPGSColor<<<gridFor(nm), B, 0, s>>>(d_, mOrder_.p, mOff_.p, col, ss, 2);
        ctl(CTL_STAB_END, vRestS, 0);
        if ((it & 15) == 15) {
          const Counters<R> cc = readCounters();
          if (cc.stabDone)
            break;
        }
      }
      KCHECK("stabilization");
    }
  }
  mark(ST_LEDGER);
  if (usePGS) {  // src/contact_preprocessing.hpp:160-192
    if (nm > 0) {
      lkeysS_.ensure(nm, false, s);
      lpermIn_.ensure(nm, false, s);
      lperm_.ensure(nm, false, s);
      const int kb = bitsFor((long)numParticles_ + 1);
      lkeysIn_.ensure(nm, false, s);
      if (!keptM_ && numParticles_ == numReal_) {  // no ghost images: the list is in real-key order
        ledFlag_.ensure((size_t)nm + 1, false, s);
        ledPos_.ensure((size_t)nm + 1, false, s);
        ++launches_, kLedgerFlags<<<gridFor(nm), B, 0, s>>>(nm, pairKeys_.p, ledFlag_.p);
        cudaCheck(cudaMemsetAsync(ledFlag_.p + nm, 0, sizeof(int), s), "memset");
        exclusiveSum(ledFlag_.p, ledPos_.p, nm + 1);
        ++launches_, kLedgerRanks<<<gridFor(nm), B, 0, s>>>(nm, kb, pairKeys_.p, ledFlag_.p, ledPos_.p, lkeysS_.p,
                                                            lperm_.p);
        KCHECK("ledger ranks");
      } else if (ledgerSplit_) {  // ghost images: sort the ghost manifolds alone, then merge
        const int nG = ledgerGhosts_;
        ledOKeys_.ensure(std::max(nG, 1), false, s);
        ledOKeysS_.ensure(std::max(nG, 1), false, s);
        ledOIdx_.ensure(std::max(nG, 1), false, s);
        ledOIdxS_.ensure(std::max(nG, 1), false, s);
        if (nG > 0) {
          ++launches_, kLedgerApart<<<gridFor(nm), B, 0, s>>>(nm, lkeysIn_.p, ledGhost_.p, ledGPos_.p, ledOKeys_.p,
                                                              ledOIdx_.p);
          sortPairs(ledOKeys_.p, ledOKeysS_.p, ledOIdx_.p, ledOIdxS_.p, nG, 2 * kb);
        }
        ++launches_, kLedgerMerge<R><<<gridFor((long)nm + nG), B, 0, s>>>(d_, nm, nG, kb, lkeysIn_.p, ledFlag_.p,
                                                                         ledPos_.p, ledGhost_.p, ledGPos_.p,
                                                                         ledOKeysS_.p, ledOIdxS_.p, lkeysS_.p,
                                                                         lperm_.p);
        KCHECK("ledger merge");
      } else if (!keptM_) {  // the ledger order depends on the manifolds' real keys only
        ++launches_, kLedgerKeys<<<gridFor(nm), B, 0, s>>>(nm, kb, pairKeys_.p, lkeysIn_.p, lpermIn_.p);
        sortPairs(lkeysIn_.p, lkeysS_.p, lpermIn_.p, lperm_.p, nm, 2 * kb);
      }
      ++launches_, kCommitLedger<<<gridFor(nm), B, 0, s>>>(d_, nm, lperm_.p);
      KCHECK("commit ledger");
    }
    prevPairCount_ = nm;
  }
  mark(ST_FRICTION);
  if (legacyFriction && nc > 0) {  // src/sim.hpp:423-429
    ++launches_, kCountFriction<<<gridFor(nc), B, 0, s>>>(d_, nc);
    qA_.ensure(nc, false, s);
    qB_.ensure(nc, false, s);
    qC_.ensure(nc, false, s);
    iC_.ensure(nc, false, s);
    ++launches_, kFrictionImpulses<<<gridFor(nc), B, 0, s>>>(d_, nc, mu_, qA_.p, qB_.p, qC_.p, iC_.p);
    buildIncidence(1, nc, numReal_);
    Incidence incF{incOff_.p, incValsS_.p};
    dVel_.zero(s);
    dAngVel_.zero(s);
    ++launches_, kFrictionGather<<<gridFor(numReal_), B, 0, s>>>(d_, numReal_, incF, qA_.p, qB_.p, qC_.p, iC_.p);
    ++launches_, kApplyVelocityDeltas<<<gridFor(numParticles_), B, 0, s>>>(d_, numParticles_);
    KCHECK("legacy friction");
  } else if (legacyFriction) {
    dVel_.zero(s);
    dAngVel_.zero(s);
  }
  mark(ST_INTEGRATE);
  if (numParticles_ > 0) {
    ++launches_, kApplyVelPredictPos<<<gridFor(numParticles_), B, 0, s>>>(d_, numParticles_, dt_);
    KCHECK("apply vel predict pos");
  }
  mark(ST_COLOR_P);
  mark(ST_POSITION);
  const R posTol = R(1e-4) * baseRadius_ * gs_;
  if (nc > 0)
    posLamC_.zero(s, nc);
  const bool posJacobi = (posLeft > 0 || !useGS_) && nc > 0;
  if (posJacobi) {
    buildIncidence(2, nc, numParticles_);
    qA_.ensure(nc, false, s);
    iC_.ensure(nc, false, s);
  }
  Incidence incP{incOff_.p, incValsS_.p};
  const bool posPersistent = useGS_ && posLeft == 0 && ncolP > 0 && posIters_ > 0;
  if (posPersistent) {
    gbar_.ensure(2, false, s);
    const GridBar gb{gbar_.p, &ctr_.p->err, barrierSleepNs_, barrierSpins_};
    ctl(CTL_POS_BEGIN, R(0), 0);
    if (batch_) {
      ++launches_, kSweepScenes<R, 2, 3><<<numScenes_, sceneBlock(), 0, s>>>(d_, sceneLpt_.p, cOrder_.p, cOff_.p, posIters_, sp, posTol);
      tuneEnd();
    }
    else if (!(nc <= sweepClusterEntries_ &&
               launchCluster(kSweepLoop<R, 2, 3, true>, d_, (const int*)cOrder_.p, (const int*)cOff_.p, ncolP,
                             posIters_, sp, posTol, gb, PgsRecs<R>{})))
      launchCoop(kSweepLoop<R, 2, 3>, d_, (const int*)cOrder_.p, (const int*)cOff_.p, ncolP, posIters_, sp, posTol, gb,
                 PgsRecs<R>{});
    KCHECK("position loop");
  }
  const bool posEmpty = useGS_ && posLeft == 0 && ncolP <= 0 && posIters_ > 0 && posTol > R(0);
  if (posEmpty) {  // as velEmpty: maxOverlap = 0 < posTol ends the loop after its first sweep
    ctl(CTL_POS_BEGIN, R(0), 0);
    ctl(CTL_POS_END, posTol, 0);
  }
  for (int it = 0; it < (posPersistent || posEmpty ? 0 : posIters_); ++it) {
    if (useGS_) {
      ctl(CTL_POS_BEGIN, R(0), 0);
      for (int col = 0; col < ncolP; ++col)
        ++launches_, kPosGSColor<<<gridFor(nc), B, 0, s>>>(d_, cOrder_.p, cOff_.p, col, 3);
      if (posLeft > 0) {
        ++launches_, kPosJacobiPre<<<gridFor(nc), B, 0, s>>>(d_, nc, 1, qA_.p, iC_.p, 3);
        ++launches_, kPosJacobiGather<<<gridFor(numParticles_), B, 0, s>>>(d_, numParticles_, incP, qA_.p, iC_.p, 3);
        ++launches_, kApplyUpdatesGated<<<gridFor(numParticles_), B, 0, s>>>(d_, numParticles_, 3);
      }
      ctl(CTL_POS_END, posTol, 0);
    } else {
      if (nc > 0) {
        ++launches_, kPosJacobiPre<<<gridFor(nc), B, 0, s>>>(d_, nc, 0, qA_.p, iC_.p, 0);
        ++launches_, kPosJacobiGather<<<gridFor(numParticles_), B, 0, s>>>(d_, numParticles_, incP, qA_.p, iC_.p, 0);
      }
      ++launches_, kApplyUpdatesGated<<<gridFor(numParticles_), B, 0, s>>>(d_, numParticles_, 0);
    }
    KCHECK("position sweep");
  }
  mark(ST_COMMIT);
  if (usePGS && nm > 0) {  // src/contact_preprocessing.hpp:501-538 (scratch = vn0, as the reference)
    ++launches_, kPosLoad<<<gridFor(nm), B, 0, s>>>(d_, nm, nc, segStart_.p, cperm_.p, dt_, vn0_.p);
    ++launches_, kPosLoadScatter<<<gridFor(nm), B, 0, s>>>(d_, nm, lperm_.p, vn0_.p);
    KCHECK("commit position impulse");
  }
  if (numReal_ > 0) {
    DomainP<R> dom;
    for (int a = 0; a < 3; ++a) {
      dom.mn[a] = dmin_[a], dom.mx[a] = dmax_[a], dom.sz[a] = dsize_[a], dom.per[a] = per_[a];
    }
    if (mixed_)
      ++launches_, kMixedCommit<<<gridFor(numReal_), B, 0, s>>>(d_, numReal_, dom, posD_.p, quatD_.p);
    else
      ++launches_, kFinalCommit<<<gridFor(numReal_), B, 0, s>>>(d_, numReal_, dom);
    KCHECK("final commit");
  }
  if (thTau_ > R(0) && dt_ > R(0) && numReal_ > 0) {  // src/integration.hpp:229-272
    thermo_.ensure(2, false, s);
    ++launches_, kThermoEnergy<<<1, 1, 0, s>>>(d_, numReal_, thermo_.p);
    double ke[2];
    readBack(ke, thermo_.p, sizeof ke);
    sync();
    const double ndof = 3.0 * numReal_, kB = (double)thKB_, tau = (double)thTau_, Tt = (double)thT_;
    auto lam = [&](double kin) -> R {
      if (ndof <= 0 || kB <= 0)
        return R(1);
      const double Tc = (2.0 * kin) / (ndof * kB);
      if (Tc < 1e-6)
        return R(1);
      double f = 1.0 + ((double)dt_ / tau) * (Tt / Tc - 1.0);
      if (f < 0.0)
        f = 0.0;
      return static_cast<R>(std::sqrt(f));
    };
    ++launches_, kThermoScale<<<gridFor(numReal_), B, 0, s>>>(d_, numReal_, lam(ke[0]), lam(ke[1]));
    KCHECK("thermostat");
  }
  mark(ST_END);
  flushMarks();
  if (prof_) {
    const Counters<R> cc = readCounters();
    sweeps_[0] += cc.velSweeps;
    sweeps_[1] += cc.stabSweeps;
    sweeps_[2] += cc.posSweeps;
    sweeps_[3] += 1;
  }
  // the colourings, orders and groupings of this substep are now the reference for the next one
  topoValid_ = useGS_;
  // no final synchronisation: the next call's launches queue behind this substep on the stream,
  // and every getter synchronises before it reads
}

// src/sim.hpp:494-541
template <class R>
R Sim<R>::computeOverlaps() {
  topoValid_ = false;  // detectAll records a contact list that no colouring follows
  if (batch_)
    batchBegin();
  const R maxRad = maxOwnedRadius();
  const R margin = R(0.1) * maxRad;
  numParticles_ = numReal_;
  cudaCheck(cudaMemcpyAsync(posPred_.p, pos_.p, capacity_ * sizeof(Q4<R>), cudaMemcpyDeviceToDevice, stream_), "D2D");
  cudaCheck(cudaMemcpyAsync(quatPred_.p, quat_.p, capacity_ * sizeof(Q4<R>), cudaMemcpyDeviceToDevice, stream_), "D2D");
  resetGhosts(maxRad);
  if (numParticles_ > 0)
    ++launches_, kRadii<<<gridFor(numParticles_), kBlock, 0, stream_>>>(d_, numParticles_, gs_, baseRadius_);
  detectAll(margin);
  numParticles_ = numReal_;
  return readCounters().maxOverlap;
}
template <class R>
int Sim<R>::numContacts() {
  return readCounters().contactCount;
}
template <class R>
int Sim<R>::numManifolds() {
  return readCounters().manifoldCount;
}
template <class R>
R Sim<R>::maxOverlap() {
  return readCounters().maxOverlap;
}

// =============================================================================================
// diagnostics
// =============================================================================================
// the last substep's sizes, colour counts, sweeps, overlap and error bits
template <class R>
void Sim<R>::lastCounters(long* sizes, int* ints, double* maxOverlap) {  // ints: 8 values
  const Counters<R> c = readCounters();
  sizes[0] = c.pairCount;
  sizes[1] = c.contactCount;
  sizes[2] = c.manifoldCount;
  ints[0] = ncolVLast_;
  ints[1] = ncolPLast_;
  ints[2] = c.velSweeps;
  ints[3] = c.stabSweeps;
  ints[4] = c.posSweeps;
  ints[5] = c.err;
  ints[6] = colorRounds_[0];
  ints[7] = colorRounds_[1];
  *maxOverlap = (double)c.maxOverlap;
}
template <class R>
void Sim<R>::counts(long* out) {
  const Counters<R> c = readCounters();
  out[0] = c.pairCount;
  out[1] = c.contactCount;
  out[2] = c.manifoldCount;
  out[3] = numParticles_;
  out[4] = prevPairCount_;
  out[5] = capacity_;
  out[6] = maxContacts_;
  out[7] = (long)pairs_.n;
}
template <class T>
static std::vector<T> d2h(const T* p, long n, cudaStream_t s) {
  std::vector<T> h(std::max(n, 0L));
  if (n > 0) {
    cudaCheck(cudaMemcpyAsync(h.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost, s), "D2H");
    cudaCheck(cudaStreamSynchronize(s), "sync");
  }
  return h;
}
template <class R>
long Sim<R>::getPairs(int* out, long cap) {
  const long n = std::min<long>(readCounters().pairCount, (long)pairs_.n);
  const auto h = d2h(pairs_.p, n, stream_);
  for (long i = 0; i < n && 2 * i + 1 < cap; ++i) {
    out[2 * i] = h[i].x;
    out[2 * i + 1] = h[i].y;
  }
  return n;
}
template <class R>
long Sim<R>::getContacts(double* out, long cap, bool muOnly) {
  const long n = readCounters().contactCount;
  const auto ab = d2h(cab_.p, n, stream_);
  const auto cn = d2h(cn_.p, n, stream_), ra = d2h(crA_.p, n, stream_), rb = d2h(crB_.p, n, stream_),
             bv = d2h(cbv_.p, n, stream_);
  for (long i = 0; i < n; ++i) {
    if (muOnly) {
      if (i < cap)
        out[i] = bv[i].w;
      continue;
    }
    if (17 * i + 16 >= cap)
      break;
    const double v[17] = {(double)ab[i].x, (double)ab[i].y, cn[i].x, cn[i].y, cn[i].z, ra[i].x, ra[i].y, ra[i].z,
                          rb[i].x, rb[i].y, rb[i].z, cn[i].w, ra[i].w, bv[i].x, bv[i].y, bv[i].z, rb[i].w};
    std::memcpy(out + 17 * i, v, sizeof v);
  }
  return n;
}
template <class R>
long Sim<R>::getManifolds(double* out, long cap) {
  const long n = readCounters().manifoldCount;
  const auto ab = d2h(mab_.p, n, stream_);
  const auto np = d2h(mnp_.p, n, stream_);
  const auto N = d2h(mN_.p, n, stream_), TA = d2h(mTA_.p, n, stream_), TB = d2h(mTB_.p, n, stream_),
             rA = d2h(mrA_.p, n, stream_), rB = d2h(mrB_.p, n, stream_), wv = d2h(mwv_.p, n, stream_);
  for (long i = 0; i < n && 23 * i + 22 < cap; ++i) {
    const double v[23] = {(double)ab[i].x, (double)ab[i].y, N[i].x,  N[i].y,  N[i].z,  TA[i].x,
                          TA[i].y,         TA[i].z,         TB[i].x, TB[i].y, TB[i].z, rA[i].x,
                          rA[i].y,         rA[i].z,         rB[i].x, rB[i].y, rB[i].z, (double)np[i],
                          wv[i].x,         wv[i].y,         wv[i].z, N[i].w,  TA[i].w};
    std::memcpy(out + 23 * i, v, sizeof v);
  }
  return n;
}
template <class R>
long Sim<R>::getColors(bool manifold, int* out, long cap) {
  const Counters<R> c = readCounters();
  const long n = manifold ? c.manifoldCount : c.contactCount;
  const auto h = d2h(manifold ? mColor_.p : cColor_.p, n, stream_);
  for (long i = 0; i < n && i < cap; ++i)
    out[i] = h[i];
  return n;
}
template <class R>
long Sim<R>::getLambda(double* out, long cap) {
  const long n = readCounters().manifoldCount;
  const auto l = d2h(lambda_.p, n, stream_);
  const auto t = d2h(lambdaT_.p, n, stream_);
  for (long i = 0; i < n && 4 * i + 3 < cap; ++i) {
    out[4 * i] = l[i];
    out[4 * i + 1] = t[i].x;
    out[4 * i + 2] = t[i].y;
    out[4 * i + 3] = t[i].z;
  }
  return n;
}
template <class R>
long Sim<R>::getPairKeys(unsigned long long* out, long cap) {
  const long n = readCounters().manifoldCount;
  const auto h = d2h(pairKeys_.p, n, stream_);
  for (long i = 0; i < n && i < cap; ++i)
    out[i] = h[i];
  return n;
}
template <class R>
long Sim<R>::getLedger(unsigned long long* keys, double* vals, long cap) {
  const long n = prevPairCount_;
  const auto k = d2h(prevKeys_.p, n, stream_);
  const auto l = d2h(prevLambda_.p, n, stream_);
  const auto t = d2h(prevLambdaT_.p, n, stream_);
  const auto p = d2h(prevPosImp_.p, n, stream_);
  for (long i = 0; i < n && i < cap; ++i) {
    keys[i] = k[i];
    vals[5 * i] = l[i];
    vals[5 * i + 1] = t[i].x;
    vals[5 * i + 2] = t[i].y;
    vals[5 * i + 3] = t[i].z;
    vals[5 * i + 4] = p[i];
  }
  return n;
}
template <class R>
long Sim<R>::getGrounded(int* out, long cap) {
  ensureGrounded();
  const long n = numReal_;
  const auto h = d2h(grounded_.p, n, stream_);
  for (long i = 0; i < n && i < cap; ++i)
    out[i] = h[i];
  return n;
}
template <class R>
long Sim<R>::getPosLambda(double* out, long cap) {
  const long n = readCounters().contactCount;
  const auto h = d2h(posLamC_.p, n, stream_);
  for (long i = 0; i < n && i < cap; ++i)
    out[i] = h[i];
  return n;
}
// test hook: shrink (or grow) the contact capacity, as replacing the reference's contact View
template <class R>
void Sim<R>::setMaxContacts(int n) {
  topoValid_ = false;
  if ((size_t)n > cab_.n)
    allocContactBuffers(n);
  maxContacts_ = n;
  refreshDev();
}

// =============================================================================================
// Hertz-Mindlin engine: src/sim.hpp:545-750
// =============================================================================================
// src/sim.hpp:597-625
template <class R>
void Sim<R>::hertzCommitHistory() {
  const int n = hzNumPairs_;
  if (n <= 0) {
    hzPrevCount_ = 0;
    return;
  }
  lpermIn_.ensure(n, false, stream_);
  lperm_.ensure(n, false, stream_);
  ++launches_, kIota<R><<<gridFor(n), kBlock, 0, stream_>>>(lpermIn_.p, n);
  sortPairs(hzKeys_.p, hzPrevKeys_.p, lpermIn_.p, lperm_.p, n, 64);
  ++launches_, kHertzGatherPrev<<<gridFor(n), kBlock, 0, stream_>>>(n, lperm_.p, hzXi_.p, hzPrevXi_.p);
  KCHECK("hertz commit history");
  hzPrevCount_ = n;
}
// src/sim.hpp:545-594
template <class R>
void Sim<R>::hertzRebuildPairs(R skin) {
  cudaCheck(cudaMemcpyAsync(posPred_.p, pos_.p, capacity_ * sizeof(Q4<R>), cudaMemcpyDeviceToDevice, stream_), "D2D");
  const int np = findCollisionsGrow(skin, posPred_.p);
  const size_t need = pairs_.n;
  if (hzXi_.n < need) {
    // fresh buffers, as the reference reallocates (the previous history was committed above)
    DBuf<u64> pk;
    DBuf<Q4<R>> px;
    pk.ensure(need, false, stream_);
    px.ensure(need, false, stream_);
    if (hzPrevCount_ > 0) {
      cudaCheck(cudaMemcpyAsync(pk.p, hzPrevKeys_.p, hzPrevCount_ * sizeof(u64), cudaMemcpyDeviceToDevice, stream_), "D2D");
      cudaCheck(cudaMemcpyAsync(px.p, hzPrevXi_.p, hzPrevCount_ * sizeof(Q4<R>), cudaMemcpyDeviceToDevice, stream_), "D2D");
    }
    sync();
    std::swap(pk.p, hzPrevKeys_.p);
    std::swap(pk.n, hzPrevKeys_.n);
    std::swap(px.p, hzPrevXi_.p);
    std::swap(px.n, hzPrevXi_.n);
    hzXi_.ensure(need, false, stream_);
    hzSnPair_.ensure(need, false, stream_);
    hzKeys_.ensure(need, false, stream_);
  }
  if (np > 0) {
    ++launches_, kHertzCarry<<<gridFor(np), kBlock, 0, stream_>>>(d_, np, hzPrevCount_, hzPrevKeys_.p, hzPrevXi_.p, hzKeys_.p,
                                                      hzXi_.p);
    KCHECK("hertz carry");
    hzSnPair_.zero(stream_, np);
  }
  hzNumPairs_ = np;
  cudaCheck(cudaMemcpyAsync(hzRefPos_.p, pos_.p, numReal_ * sizeof(Q4<R>), cudaMemcpyDeviceToDevice, stream_), "D2D");
  // pair incidence per body (pair order), reused until the next rebuild
  buildIncidence(3, np, numReal_);
}
// src/solver_hertz.hpp:343-370
template <class R>
int Sim<R>::hertzWallCandidates(R skin) {
  const int n = numReal_;
  iC_.ensure(n + 1, false, stream_);
  iD_.ensure(n + 1, false, stream_);
  iC_.zero(stream_, n + 1);
  ++launches_, kHertzWallCand<R, 0><<<gridFor(n), kBlock, 0, stream_>>>(d_, n, (int)wallsHost_.size(), skin, iC_.p, nullptr,
                                                           nullptr, 0);
  exclusiveSum(iC_.p, iD_.p, n + 1);
  int total = 0;
  cudaCheck(cudaMemcpyAsync(&total, iD_.p + n, sizeof(int), cudaMemcpyDeviceToHost, stream_), "D2H");
  sync();
  const int cap = (int)hzWallCand_.n;
  ++launches_, kHertzWallCand<R, 1><<<gridFor(n), kBlock, 0, stream_>>>(d_, n, (int)wallsHost_.size(), skin, nullptr, iD_.p,
                                                           hzWallCand_.p, cap);
  KCHECK("hertz wall candidates");
  hzCandOff_.ensure(n + 1, false, stream_);
  cudaCheck(cudaMemcpyAsync(hzCandOff_.p, iD_.p, (n + 1) * sizeof(int), cudaMemcpyDeviceToDevice, stream_), "D2D");
  return total < cap ? total : cap;
}
// src/sim.hpp:628-750
template <class R>
void Sim<R>::stepHertz(R dt, int nsteps, R skinFrac) {
  dt_ = dt;
  topoValid_ = false;
  if (batch_)
    throw std::runtime_error("step_hertz: not supported for batched scenes");
  if (mixed_)
    throw std::runtime_error("step_hertz: not supported in the FP32-mixed precision");
  if (per_[0] || per_[1] || per_[2])
    throw std::runtime_error("step_hertz: periodic domains not supported");
  if (!planesHost_.empty())
    throw std::runtime_error("step_hertz: analytic planes not supported (use an SDF wall)");
  if ((int)wallsHost_.size() > kHertzMaxWalls)
    throw std::runtime_error("step_hertz: too many SDF walls");
  const int n = numReal_;
  if (n > 0)
    ++launches_, kRadii<<<gridFor(n), kBlock, 0, stream_>>>(d_, n, gs_, baseRadius_);
  // min radius = min over scale * gs * bR: rounding is monotone, so it is minScale * gs * bR
  R minRad = std::numeric_limits<R>::max();
  if (n > 0) {
    const auto sc = [&] {
      std::vector<R> h(n);
      cudaCheck(cudaMemcpyAsync(h.data(), rad_.p, n * sizeof(R), cudaMemcpyDeviceToHost, stream_), "D2H");
      sync();
      return h;
    }();
    for (R r : sc)
      if (r < minRad)
        minRad = r;
  }
  const R skin = skinFrac * minRad;
  const R rebuildAt = R(0.25) * skin * skin;
  bool rebuild = hzNumPairs_ < 0;
  if (!rebuild)  // the incidence buffers are shared with the XPBD step: rebuild them for this call
    buildIncidence(3, hzNumPairs_, numReal_);
  const bool hasShapes = shape_.numPoints > 0;
  const int nw = (int)wallsHost_.size();
  HertzP<R> P{dt, eN_, mu_, gs_, hzContactFrac_, nw};
  const V3<R> g{g_[0], g_[1], g_[2]};
  for (int k = 0; k < nsteps; ++k) {
    if (rebuild) {
      mark(ST_HERTZ_REBUILD);
      hertzCommitHistory();
      hertzRebuildPairs(skin);
      if (nw > 0)
        hzNumWallCand_ = hertzWallCandidates(skin);
      rebuild = false;
    }
    mark(ST_HERTZ_PAIRS);
    const int np = hzNumPairs_;
    qA_.ensure(std::max(np, 1), false, stream_);
    qB_.ensure(std::max(np, 1), false, stream_);
    qC_.ensure(std::max(np, 1), false, stream_);
    iE_.ensure(std::max(np, 1), false, stream_);
    if (np > 0) {
      if (hasShapes)
        ++launches_, kHertzShapePairs<<<gridFor(np), kBlock, 0, stream_>>>(d_, np, P, hzXi_.p, hzSnPair_.p, qA_.p, qB_.p, qC_.p,
                                                               iE_.p);
      else
        ++launches_, kHertzPairs<<<gridFor(np), kBlock, 0, stream_>>>(d_, np, P, hzXi_.p, qA_.p, qB_.p, qC_.p, iE_.p);
      KCHECK("hertz pairs");
    }
    const int nc = (nw > 0) ? hzNumWallCand_ : 0;
    hzFW_.ensure(std::max(nc, 1), false, stream_);
    hzTW_.ensure(std::max(nc, 1), false, stream_);
    hzOnW_.ensure(std::max(nc, 1), false, stream_);
    if (nc > 0) {
      ++launches_, kHertzWalls<<<gridFor(nc), kBlock, 0, stream_>>>(d_, nc, P, hzWallCand_.p, hzXiWall_.p, hzSnWall_.p,
                                                        hasShapes ? 1 : 0, hzFW_.p, hzTW_.p, hzOnW_.p);
      KCHECK("hertz walls");
    }
    mark(ST_HERTZ_INTEGRATE);
    if (n > 0) {
      ++launches_, kHertzGatherIntegrate<<<gridFor(n), kBlock, 0, stream_>>>(
          d_, n, incOff_.p, incValsS_.p, qA_.p, qB_.p, qC_.p, iE_.p, nc > 0 ? hzCandOff_.p : nullptr, nc, hzFW_.p,
          hzTW_.p, hzOnW_.p, g, dt, hasShapes ? 1 : 0);
      KCHECK("hertz integrate");
    }
    if ((k & 15) == 15 || k == nsteps - 1) {
      rA_.ensure(1, false, stream_);
      rA_.zero(stream_, 1);
      if (n > 0)
        ++launches_, kHertzMaxDisp2<<<gridFor(n), kBlock, 0, stream_>>>(d_, n, hzRefPos_.p, rA_.p);
      R m = 0;
      cudaCheck(cudaMemcpyAsync(&m, rA_.p, sizeof(R), cudaMemcpyDeviceToHost, stream_), "D2H");
      sync();
      if (n <= 0)
        m = std::numeric_limits<R>::lowest();
      if (m > rebuildAt)
        rebuild = true;
    }
  }
  mark(ST_END);
  flushMarks();
  cudaCheck(cudaMemcpyAsync(posPred_.p, pos_.p, capacity_ * sizeof(Q4<R>), cudaMemcpyDeviceToDevice, stream_), "D2D");
  cudaCheck(cudaMemcpyAsync(velPred_.p, vel_.p, capacity_ * sizeof(Q4<R>), cudaMemcpyDeviceToDevice, stream_), "D2D");
  sync();
}
template <class R>
long Sim<R>::getHertz(unsigned long long* keys, double* xi, long cap) {
  const long n = std::max(hzNumPairs_, 0);
  const auto k = d2h(hzKeys_.p, n, stream_);
  const auto x = d2h(hzXi_.p, n, stream_);
  for (long i = 0; i < n && i < cap; ++i) {
    keys[i] = k[i];
    xi[3 * i] = x[i].x;
    xi[3 * i + 1] = x[i].y;
    xi[3 * i + 2] = x[i].z;
  }
  return n;
}

// ---- support levels (src/contact_preprocessing.hpp:213-253), evaluated lazily ----
// Each substep of the PGS path decays every level by 8 and then runs 8 serial sweeps over that
// substep's support graph. A level is at most 255, so anything older than 32 logged substeps has
// decayed to 0: the levels are a function of the last 32 support graphs alone. They are read only
// by the one-sided stabilization pass, so each substep just records its graph in a 32-slot ring and
// the sweeps are replayed (from the last checkpoint, or from zero over the last 32 graphs) only when
// the pass needs the levels. The result is identical to sweeping every substep.
// get_sdf_grid (src/sim.hpp:1538-1542, src/output_sdf.hpp:25-196), flat x-fastest
template <class R>
std::vector<R> Sim<R>::sdfGrid(int rx, int ry, int rz) {
  if (rx < 1 || ry < 1 || rz < 1)
    throw std::invalid_argument("get_sdf_grid: resolution must be positive");
  cudaStream_t s = stream_;
  const long total = (long)rx * ry * rz;
  SdfGridP<R> G;
  G.rx = rx, G.ry = ry, G.rz = rz;
  G.px = per_[0], G.py = per_[1], G.pz = per_[2];
  const int res[3] = {rx, ry, rz};
  for (int a = 0; a < 3; ++a) {
    G.o[a] = dmin_[a];
    G.vox[a] = (dmax_[a] - dmin_[a]) / R(res[a]);
  }
  sdfA_.ensure(total, false, s);
  sdfB_.ensure(total, false, s);
  sdfState_.ensure(total, false, s);
  ++launches_, kSdfInit<<<gridFor(total), kBlock, 0, s>>>(sdfA_.p, sdfState_.p, total);
  if (numReal_ > 0)
    ++launches_, kSdfSplat<<<gridFor(32L * numReal_, 128), 128, 0, s>>>(d_, numReal_, G, sdfA_.p, sdfState_.p);
  const int iters = std::max(std::max(rx, ry), rz) * 4;
  R* in = sdfA_.p;
  R* out = sdfB_.p;
  for (int it = 0; it < iters; ++it) {
    ++launches_, kSdfEikonal<<<gridFor(total), kBlock, 0, s>>>(G, in, out, sdfState_.p, G.vox[0]);
    std::swap(in, out);
  }
  KCHECK("sdf grid");
  std::vector<R> h(total);
  cudaCheck(cudaMemcpyAsync(h.data(), in, total * sizeof(R), cudaMemcpyDeviceToHost, s), "D2H");
  sync();
  return h;
}

// "ordered" stabilization (src/sim.hpp:357-400): fresh height levels, manifolds bucketed by
// (level, colour), symmetric sweeps bottom-up then top-down until the residual drains
// the multilevel pass (src/sim.hpp:303-356): the hierarchy, then the smoothing / coarse loop,
// driven from the host (pdem_multilevel.cuh)
template <class R>
void Sim<R>::multilevelStabilization(int nm, int ncol, const SolveP<R>& ss, R vRestS, R gMag) {
  cudaStream_t s = stream_;
  const int B = kBlock;
  const int nr = numReal_;
  if (nm <= 0 || nr <= 0)
    return;
  const R qsThr = R(8) * dt_ * gMag;
  const int parentCap = 5 * capacity_, groupCap = 4 * capacity_;
  mlPacked_.ensure(nm, false, s);
  mlParent_.ensure(parentCap, false, s);
  mlGrp_.ensure(nr, false, s);
  mlMate_.ensure(nr, false, s);
  mlFlag_.ensure((size_t)nr + 1, false, s);
  mlPos_.ensure((size_t)nr + 1, false, s);
  mlWin_.ensure(nr, false, s);
  mlMask_.ensure(nr, false, s);
  mlMassG_.ensure(groupCap, false, s);
  mlInvMassG_.ensure(groupCap, false, s);
  mlVelG_.ensure(groupCap, false, s);
  mlVelG0_.ensure(groupCap, false, s);
  mlInt_.ensure(2, false, s);
  mlQS_.ensure(1, false, s);
  cudaCheck(cudaMemsetAsync(mlPacked_.p, 0xff, nm * sizeof(long long), s), "memset");  // every slot 63
  ++launches_, kMlIota<<<gridFor(nr), B, 0, s>>>(mlGrp_.p, nr);
  struct Level {
    int groupOff, numGroups, parentOff, numColors;
  };
  std::vector<Level> H;
  auto readInt = [&](const int* dev) {
    int v = 0;
    cudaCheck(cudaMemcpyAsync(&v, dev, sizeof v, cudaMemcpyDeviceToHost, s), "D2H");
    sync();
    return v;
  };
  int ngPrev = nr, parentOff = 0, groupOff = 0;
  for (int lvl = 1; lvl <= kMlMaxLevels; ++lvl) {  // src/solver_multilevel.hpp:154-322
    if (parentOff + ngPrev > parentCap)
      break;
    cudaCheck(cudaMemsetAsync(mlWin_.p, 0xff, ngPrev * sizeof(long long), s), "memset");
    ++launches_, kMlMatchContend<<<gridFor(nm), B, 0, s>>>(d_, nm, qsThr, mlGrp_.p, mlWin_.p);
    ++launches_, kMlIota<<<gridFor(ngPrev), B, 0, s>>>(mlMate_.p, ngPrev);
    ++launches_, kMlMatchCommit<<<gridFor(nm), B, 0, s>>>(d_, nm, qsThr, mlGrp_.p, mlWin_.p, mlMate_.p);
    ++launches_, kMlLeader<<<gridFor(ngPrev), B, 0, s>>>(mlMate_.p, ngPrev, mlFlag_.p);
    cudaCheck(cudaMemsetAsync(mlFlag_.p + ngPrev, 0, sizeof(int), s), "memset");
    exclusiveSum(mlFlag_.p, mlPos_.p, ngPrev + 1);
    ++launches_, kMlParent<<<gridFor(ngPrev), B, 0, s>>>(mlMate_.p, mlFlag_.p, mlPos_.p, ngPrev,
                                                         mlParent_.p + parentOff);
    KCHECK("multilevel matching");
    const int ngNew = readInt(mlPos_.p + ngPrev);
    if (ngNew >= ngPrev || ngNew > (9 * ngPrev) / 10)
      break;
    if (groupOff + ngNew > groupCap)
      break;
    ++launches_, kMlCompose<<<gridFor(nr), B, 0, s>>>(mlGrp_.p, nr, mlParent_.p + parentOff);
    ++launches_, kMlGroupMass<<<1, 1, 0, s>>>(d_, nr, mlGrp_.p, mlMassG_.p + groupOff, mlInvMassG_.p + groupOff, ngNew);
    const int shift = 6 * (lvl - 1);
    cudaCheck(cudaMemsetAsync(mlMask_.p, 0, ngNew * sizeof(u64), s), "memset");
    int remaining = 1, prevRemaining = -1;
    for (int round = 0; round < 64 && remaining > 0; ++round) {
      cudaCheck(cudaMemsetAsync(mlWin_.p, 0xff, ngNew * sizeof(long long), s), "memset");
      ++launches_, kMlColorContend<<<gridFor(nm), B, 0, s>>>(d_, nm, qsThr, mlGrp_.p, mlPacked_.p, shift, mlWin_.p);
      cudaCheck(cudaMemsetAsync(mlInt_.p, 0, sizeof(int), s), "memset");
      ++launches_, kMlColorCommit<<<gridFor(nm), B, 0, s>>>(d_, nm, qsThr, mlGrp_.p, mlPacked_.p, shift, mlWin_.p,
                                                            mlMask_.p, mlInt_.p);
      KCHECK("multilevel colouring");
      const int rem = readInt(mlInt_.p);
      if (rem == prevRemaining)
        break;
      prevRemaining = rem;
      remaining = rem;
    }
    cudaCheck(cudaMemsetAsync(mlInt_.p + 1, 0xff, sizeof(int), s), "memset");  // -1
    ++launches_, kMlMaxColor<<<gridFor(nm), B, 0, s>>>(mlPacked_.p, nm, shift, mlInt_.p + 1);
    const int maxc = readInt(mlInt_.p + 1);
    H.push_back(Level{groupOff, ngNew, parentOff, maxc + 1});
    parentOff += ngPrev;
    groupOff += ngNew;
    ngPrev = ngNew;
    if (ngNew <= 32)
      break;
  }
  for (int it = 0; it < 2 * velIters_; ++it) {  // src/sim.hpp:337-355
    mlQS_.zero(s);
    for (int col = 0; col < ncol; ++col)
      ++launches_, kPGSColorQS<<<gridFor(nm), B, 0, s>>>(d_, mOrder_.p, mOff_.p, col, ss, mlQS_.p);
    if (!H.empty()) {  // src/solver_multilevel.hpp:331-478
      ++launches_, kMlIota<<<gridFor(nr), B, 0, s>>>(mlGrp_.p, nr);
      for (size_t l = 0; l < H.size(); ++l) {
        const Level& L = H[l];
        const int shift = 6 * (int)l;
        ++launches_, kMlCompose<<<gridFor(nr), B, 0, s>>>(mlGrp_.p, nr, mlParent_.p + L.parentOff);
        ++launches_, kMlRestrict<<<1, 1, 0, s>>>(d_, nr, mlGrp_.p, mlVelG_.p + L.groupOff, mlVelG0_.p + L.groupOff,
                                                 mlMassG_.p + L.groupOff, L.numGroups);
        for (int sw = 0; sw < 2; ++sw)
          for (int color = 0; color < L.numColors; ++color)
            ++launches_, kMlCoarsePGS<<<gridFor(nm), B, 0, s>>>(d_, nm, mlGrp_.p, mlPacked_.p, shift, color,
                                                                mlVelG_.p + L.groupOff, mlInvMassG_.p + L.groupOff,
                                                                mlQS_.p);
        ++launches_, kMlProlong<<<gridFor(nr), B, 0, s>>>(d_, nr, mlGrp_.p, mlVelG_.p + L.groupOff,
                                                          mlVelG0_.p + L.groupOff);
      }
    }
    KCHECK("multilevel cycle");
    R qs = 0;
    cudaCheck(cudaMemcpyAsync(&qs, mlQS_.p, sizeof qs, cudaMemcpyDeviceToHost, s), "D2H");
    sync();
    if (qs <= vRestS)
      break;
  }
}

template <class R>
void Sim<R>::orderedStabilization(int nm, V3<R> gHat, const SolveP<R>& ss, R vRestS) {
  cudaStream_t s = stream_;
  const int B = kBlock;
  if (nm <= 0 || numReal_ <= 0)
    return;
  heights_.ensure(numReal_, false, s);
  ordChanged_.ensure(1, false, s);
  ++launches_, kHeightInit<<<gridFor(numReal_), B, 0, s>>>(heights_.p, numReal_);
  // sweeps until none changes a level (at most 1024, as the reference); four per host check,
  // which cannot change the result: a sweep at the fixed point changes nothing
  for (int sweep = 0; sweep < 1024; sweep += 4) {
    ordChanged_.zero(s);
    for (int q = 0; q < 4; ++q)
      ++launches_, kHeightSweep<<<gridFor(nm), B, 0, s>>>(d_, nm, gHat, heights_.p, ordChanged_.p);
    int changed = 0;
    cudaCheck(cudaMemcpyAsync(&changed, ordChanged_.p, sizeof changed, cudaMemcpyDeviceToHost, s), "D2H");
    sync();
    if (changed == 0)
      break;
  }
  ordKeysIn_.ensure(nm, false, s);
  ordKeys_.ensure(nm, false, s);
  ordPermIn_.ensure(nm, false, s);
  ordPerm_.ensure(nm, false, s);
  ++launches_, kLevelKeys<<<gridFor(nm), B, 0, s>>>(d_, nm, heights_.p, ordKeysIn_.p, ordPermIn_.p);
  sortPairs(ordKeysIn_.p, ordKeys_.p, ordPermIn_.p, ordPerm_.p, nm, 31);
  std::vector<int> keys(nm);
  cudaCheck(cudaMemcpyAsync(keys.data(), ordKeys_.p, nm * sizeof(int), cudaMemcpyDeviceToHost, s), "D2H");
  sync();
  std::vector<std::pair<int, int>> buckets;
  for (int b = 0; b < nm && keys[b] != INT_MAX;) {
    int e = b + 1;
    while (e < nm && keys[e] == keys[b])
      ++e;
    buckets.emplace_back(b, e);
    b = e;
  }
  const int nb = (int)buckets.size();
  for (int it = 0; it < 2 * velIters_; ++it) {
    ctl(CTL_STAB_BEGIN, R(0), 0);
    for (int pass = 0; pass < 2; ++pass)
      for (int q = 0; q < nb; ++q) {
        const auto [b, e] = buckets[pass == 0 ? q : nb - 1 - q];
        ++launches_, kPGSBucket<<<gridFor(e - b), B, 0, s>>>(d_, ordPerm_.p, b, e - b, keys[b] % 64, ss, 2);
      }
    ctl(CTL_STAB_END, vRestS, 0);
    if (readCounters().stabDone)
      break;
  }
  KCHECK("ordered stabilization");
}

template <class R>
void Sim<R>::logSupportGraph(int nm, V3<R> gHat) {
  const int slot = (int)(gLog_ % kGroundRing);
  gRingNm_[slot] = nm;
  gRingReal_[slot] = numReal_;
  gRingScenes_[slot] = batch_ ? numScenes_ : 0;
  if (batch_) {  // the scenes' edge ranges of this substep, for one warp per scene at replay
    if (gRingScn_[slot].n < (size_t)numScenes_ + 1)
      for (auto& b : gRingScn_)
        b.ensure(numScenes_ + 1, false, stream_);
    cudaCheck(cudaMemcpyAsync(gRingScn_[slot].p, sceneManFirstD_.p, (numScenes_ + 1) * sizeof(int),
                              cudaMemcpyDeviceToDevice, stream_), "D2D scene ranges");
  }
  if (nm > 0) {
    // all slots grow together (and with headroom): a slot first used, or outgrown, later in a
    // run would otherwise stall a substep on cudaMalloc / cudaFree
    if (gRing_[slot].n < (size_t)nm) {
      const size_t cap = (size_t)nm + (size_t)nm / 4;
      for (auto& b : gRing_)
        b.ensure(cap, false, stream_);
    }
    ++launches_, kGroundEdges<<<gridFor(nm), kBlock, 0, stream_>>>(d_, nm, gHat, gRing_[slot].p);
    KCHECK("support graph");
  }
  ++gLog_;
}
template <class R>
void Sim<R>::ensureGrounded() {
  long pending = gLog_ - gCheckpoint_;
  if (pending <= 0)
    return;
  long start = gCheckpoint_;
  if (pending > kGroundRing) {
    start = gLog_ - kGroundRing;
    const int nr = gRingReal_[start % kGroundRing];
    if (nr > 0)
      cudaCheck(cudaMemsetAsync(grounded_.p, 0, nr, stream_), "memset");
  }
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(kGroundSweeps, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(kGroundSweepsScenes, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(kGroundLevels, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr = true;
  }
  for (long e = start; e < gLog_; ++e) {
    const int slot = (int)(e % kGroundRing);
    const int nr = gRingReal_[slot], nm = gRingNm_[slot];
    if (nr <= 0)
      continue;
    ++launches_, kGroundDecay<<<gridFor(nr), kBlock, 0, stream_>>>(d_, nr, 8);
    if (nm > 0 && gRingScenes_[slot] > 0) {
      const int S = gRingScenes_[slot];
      const bool smem = (size_t)maxSceneBodies_ * sizeof(int) <= 200 * 1024;
      if (!smem)
        gscratch_.ensure(nr, false, stream_);
      ++launches_, kGroundSweepsScenes<<<S, 32, smem ? maxSceneBodies_ * sizeof(int) : 0, stream_>>>(
          gRingScn_[slot].p, sceneFirstD_.p, 8, gRing_[slot].p, grounded_.p, gscratch_.p, smem);
    } else if (nm > 0 && (size_t)nr * 12 + (size_t)nm * 8 <= 200 * 1024 && nr < (1 << 30)) {
      ++launches_, kGroundLevels<<<1, kGroundBlock, (size_t)nr * 12 + (size_t)nm * 8, stream_>>>(
          nm, nr, 8, gRing_[slot].p, grounded_.p);
    } else if (nm > 0) {
      const bool smem = (size_t)nr * sizeof(int) <= 200 * 1024;
      if (!smem)
        gscratch_.ensure(nr, false, stream_);
      ++launches_, kGroundSweeps<<<1, 32, smem ? nr * sizeof(int) : 0, stream_>>>(nm, nr, 8, gRing_[slot].p,
                                                                                grounded_.p, gscratch_.p, smem);
    }
    KCHECK("support sweeps");
  }
  gCheckpoint_ = gLog_;
}

// ---- instrumentation ----
template <class R>
void Sim<R>::profileEnable(bool on) {
  reuse_[0] = reuse_[1] = reuse_[2] = 0;
  rankStats_[0] = rankStats_[1] = 0;
  prof_ = on;
  for (int i = 0; i < ST_COUNT; ++i) {
    stageMs_[i] = 0;
    stageHostMs_[i] = 0;
    stageCalls_[i] = 0;
  }
  launches_ = 0;
  for (long& v : sweeps_)
    v = 0;
}
template <class R>
void Sim<R>::mark(int stage) {
  if (!prof_)
    return;
  cudaEvent_t e;
  if (evFree_.empty())
    cudaCheck(cudaEventCreate(&e), "cudaEventCreate");
  else {
    e = evFree_.back();
    evFree_.pop_back();
  }
  cudaCheck(cudaEventRecord(e, stream_), "cudaEventRecord");
  const double now = std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
  marks_.push_back({stage, e, now});
}
template <class R>
void Sim<R>::timerStart() {
  if (!tStart_) {
    cudaCheck(cudaEventCreate(&tStart_), "cudaEventCreate");
    cudaCheck(cudaEventCreate(&tStop_), "cudaEventCreate");
  }
  cudaCheck(cudaEventRecord(tStart_, stream_), "cudaEventRecord");
}
template <class R>
double Sim<R>::timerStop() {
  if (!tStart_)
    return 0.0;
  cudaCheck(cudaEventRecord(tStop_, stream_), "cudaEventRecord");
  cudaCheck(cudaEventSynchronize(tStop_), "cudaEventSynchronize");
  float ms = 0;
  cudaCheck(cudaEventElapsedTime(&ms, tStart_, tStop_), "cudaEventElapsedTime");
  return ms;
}
template <class R>
void Sim<R>::flushMarks() {
  if (marks_.empty())
    return;
  sync();
  for (size_t k = 0; k + 1 < marks_.size(); ++k) {
    float ms = 0;
    cudaCheck(cudaEventElapsedTime(&ms, marks_[k].ev, marks_[k + 1].ev), "cudaEventElapsedTime");
    stageMs_[marks_[k].stage] += ms;
    stageHostMs_[marks_[k].stage] += 1e3 * (marks_[k + 1].host - marks_[k].host);
    stageCalls_[marks_[k].stage] += 1;
  }
  for (auto& m : marks_)
    evFree_.push_back(m.ev);
  marks_.clear();
}

// =============================================================================================
// FP32-mixed form: single-precision step, FP64 master positions and orientations
// =============================================================================================
template <class R>
void Sim<R>::setMixed(bool on) {
  mixed_ = on;
  if (on) {
    posD_.ensure(capacity_, false, stream_);
    quatD_.ensure(capacity_, false, stream_);
  }
}
// field 0: positions (n x 3), 2: quaternions (n x 4, x y z w); also resets the orientations to
// identity when the positions are set (set_positions resets every other field)
template <class R>
void Sim<R>::setMaster(int field, const double* a, int n) {
  if (!mixed_)
    return;
  const int m = std::min(numReal_, n);
  if (m <= 0)
    return;
  const int cols = field == 2 ? 4 : 3;
  std::vector<Q4<double>> h(m);
  for (int i = 0; i < m; ++i)
    h[i] = Q4<double>{a[cols * i], a[cols * i + 1], a[cols * i + 2], cols == 4 ? a[cols * i + 3] : 0.0};
  cudaCheck(cudaMemcpyAsync(field == 2 ? quatD_.p : posD_.p, h.data(), m * sizeof(Q4<double>),
                            cudaMemcpyHostToDevice, stream_), "H2D master");
  if (field == 0) {
    std::vector<Q4<double>> q(m, Q4<double>{0, 0, 0, 1});
    cudaCheck(cudaMemcpyAsync(quatD_.p, q.data(), m * sizeof(Q4<double>), cudaMemcpyHostToDevice, stream_), "H2D");
  }
  sync();
}
template <class R>
bool Sim<R>::getMaster(int field, double* out, long cap) {
  if (!mixed_ || (field != 0 && field != 2))
    return false;
  const int n = numReal_;
  std::vector<Q4<double>> h(std::max(n, 0));
  if (n > 0) {
    cudaCheck(cudaMemcpyAsync(h.data(), field == 2 ? quatD_.p : posD_.p, n * sizeof(Q4<double>),
                              cudaMemcpyDeviceToHost, stream_), "D2H master");
    sync();
  }
  const int cols = field == 2 ? 4 : 3;
  for (int i = 0; i < n && (long)cols * i + cols - 1 < cap; ++i) {
    out[cols * i] = h[i].x;
    out[cols * i + 1] = h[i].y;
    out[cols * i + 2] = h[i].z;
    if (cols == 4)
      out[cols * i + 3] = h[i].w;
  }
  return true;
}

// =============================================================================================
// batched form
// =============================================================================================
template <class R>
void Sim<R>::ctl(int op, R thr, int mode) {
  if (batch_)
    ++launches_, kCtlScenes<<<1, 1024, 0, stream_>>>(ctr_.p, scn_.p, numScenes_, op, thr, mode);
  else
    ++launches_, kCtl<<<1, 1, 0, stream_>>>(ctr_.p, op, thr, mode);
}
// ---- launch shape autotuner of the per-scene sweep loops (batched form) ----
// The block size of kSweepScenes does not change any result (a colour class is an independent set;
// the saturated colour runs on one thread), so it is tuned online: the first kTuneRounds x
// candidates batched substeps cycle through the candidate sizes, timing the main velocity and
// position sweep loops with events; the fastest size then stays. PDEM_SCENE_BLOCK fixes a size
// and turns the tuning off.
template <class R>
int Sim<R>::sceneBlock() const {
  return tuning_ ? kTuneBlocks[tuneStep_ % kTuneCands] : sceneBlock_;
}
template <class R>
void Sim<R>::tuneBegin() {
  if (!tuning_)
    return;
  if (!tuneEv_[0][0])
    for (auto& pr : tuneEv_)
      for (auto& e : pr)
        cudaCheck(cudaEventCreate(&e), "event");
  const int slot = tuneStep_ % (kTuneCands * kTuneRounds);
  cudaCheck(cudaEventRecord(tuneEv_[slot][0], stream_), "event");
  tuneOpen_ = true;
}
template <class R>
void Sim<R>::tuneEnd() {
  if (!tuning_ || !tuneOpen_)
    return;
  tuneOpen_ = false;
  const int slot = tuneStep_ % (kTuneCands * kTuneRounds);
  cudaCheck(cudaEventRecord(tuneEv_[slot][1], stream_), "event");
  if (++tuneStep_ < kTuneCands * kTuneRounds)
    return;
  sync();
  float best = 0;
  for (int c = 0; c < kTuneCands; ++c) {
    float tot = 0;
    for (int r = 0; r < kTuneRounds; ++r) {
      float ms = 0;
      cudaCheck(cudaEventElapsedTime(&ms, tuneEv_[r * kTuneCands + c][0], tuneEv_[r * kTuneCands + c][1]), "event");
      tot += ms;
    }
    tuneMs_[c] = tot / kTuneRounds;
    if (c == 0 || tot < best) {
      best = tot;
      sceneBlock_ = kTuneBlocks[c];
    }
  }
  tuning_ = false;
}

template <class R>
void Sim<R>::setScenes(int S, const int* first) {
  if (S < 1 || S > 1023)
    throw std::invalid_argument("set_scenes: between 1 and 1023 scenes");
  if (first[0] != 0 || first[S] != numReal_)
    throw std::invalid_argument("set_scenes: scene ranges must start at 0 and end at the particle count");
  for (int s = 0; s < S; ++s)
    if (first[s + 1] < first[s])
      throw std::invalid_argument("set_scenes: scene ranges must be non-decreasing");
  ensureGrounded();  // the logged support graphs index the previous scene layout
  bvhValid_ = false;  // the tree's leaf order must put every scene in one subtree
  topoValid_ = false;
  vValid_ = false;
  numScenes_ = S;
  sceneFirstHost_.assign(first, first + S + 1);
  if (const char* e = std::getenv("PDEM_SCENE_BLOCK")) {
    sceneBlock_ = std::max(32, std::min(kSceneBlockMax, (int)std::strtol(e, nullptr, 10) / 32 * 32));
    tuning_ = false;
  } else {
    tuning_ = true;
    tuneStep_ = 0;
  }
  maxSceneBodies_ = 0;
  for (int s = 0; s < S; ++s)
    maxSceneBodies_ = std::max(maxSceneBodies_, first[s + 1] - first[s]);
  std::vector<int> of(std::max(numReal_, 1), 0);
  for (int s = 0; s < S; ++s)
    for (int i = first[s]; i < first[s + 1]; ++i)
      of[i] = s;
  sceneOf_.ensure(capacity_, false, stream_);
  cudaCheck(cudaMemcpyAsync(sceneOf_.p, of.data(), numReal_ * sizeof(int), cudaMemcpyHostToDevice, stream_), "H2D");
  sceneFirstD_.ensure(S + 1, false, stream_);
  cudaCheck(cudaMemcpyAsync(sceneFirstD_.p, first, (S + 1) * sizeof(int), cudaMemcpyHostToDevice, stream_), "H2D");
  // the per-scene sweep loops dispatch scenes largest first (longest-processing-time order): a
  // large scene left to the last wave of blocks would set the kernel's tail
  std::vector<int> lpt(S);
  for (int k = 0; k < S; ++k)
    lpt[k] = k;
  std::stable_sort(lpt.begin(), lpt.end(),
                   [&](int a, int b) { return first[a + 1] - first[a] > first[b + 1] - first[b]; });
  sceneLpt_.ensure(std::max(S, 1), false, stream_);
  cudaCheck(cudaMemcpyAsync(sceneLpt_.p, lpt.data(), S * sizeof(int), cudaMemcpyHostToDevice, stream_), "H2D");
  scn_.ensure(S, false, stream_);
  scn_.zero(stream_, S);
  sceneParams_.ensure(3 * (size_t)S, false, stream_);
  sceneMaxScale_.ensure(S, false, stream_);
  sceneManFirstD_.ensure(S + 1, false, stream_);
  sceneConFirstD_.ensure(3 * ((size_t)S + 1), false, stream_);
  sceneLeafFirstD_.ensure(S + 1, false, stream_);
  sceneWallOffD_.ensure(S + 1, false, stream_);
  sceneE_.assign(S, eN_);
  sceneMu_.assign(S, mu_);
  batch_ = true;
  sceneParamsDirty_ = sceneWallsDirty_ = true;
  refreshDev();
  sync();
}
template <class R>
void Sim<R>::setSceneMaterial(int scene, R e, R mu) {
  if (!batch_ || scene < 0 || scene >= numScenes_)
    throw std::invalid_argument("set_scene_material: scene index out of range");
  sceneE_[scene] = e;
  sceneMu_[scene] = mu;
  sceneParamsDirty_ = true;
  maxScaleValid_ = false;
  vValid_ = false;
}
template <class R>
void Sim<R>::setWallScene(int wall, int scene) {
  if (wall < 0 || wall >= (int)wallsHost_.size())
    throw std::invalid_argument("set_wall_scene: wall index out of range");
  if (scene < -1)
    throw std::invalid_argument("set_wall_scene: scene index out of range");
  wallScene_.resize(wallsHost_.size(), -1);
  wallScene_[wall] = scene;
  sceneWallsDirty_ = true;
}
// per scene: max overlap, max approach, velocity / stabilization / position sweeps of the last substep
template <class R>
long Sim<R>::sceneCounters(double* out, long cap) {
  if (!batch_)
    return 0;
  std::vector<SceneCtl<R>> h(numScenes_);
  cudaCheck(cudaMemcpyAsync(h.data(), scn_.p, numScenes_ * sizeof(SceneCtl<R>), cudaMemcpyDeviceToHost, stream_), "D2H");
  sync();
  long k = 0;
  for (int s = 0; s < numScenes_ && k + 5 <= cap; ++s) {
    out[k++] = h[s].maxOverlap;
    out[k++] = h[s].maxApproach;
    out[k++] = h[s].velSweeps;
    out[k++] = h[s].stabSweeps;
    out[k++] = h[s].posSweeps;
  }
  return numScenes_;
}
// start of a batched substep: per-scene margins (0.1 x the scene's largest radius, as
// src/sim.hpp:61-70 computes for a scene alone), materials, wall lists and loop state
template <class R>
void Sim<R>::batchBegin() {
  if (per_[0] || per_[1] || per_[2])
    throw std::runtime_error("batched scenes: periodic domains are not supported");
  if (gf_ > R(0) || (thTau_ > R(0)))
    throw std::runtime_error("batched scenes: growth and the thermostat are not supported");
  if (!useGS_)
    throw std::runtime_error("batched scenes: the Jacobi velocity solve is not supported");
  const int S = numScenes_;
  if (sceneWallsDirty_) {
    wallScene_.resize(wallsHost_.size(), -1);
    std::vector<int> off(S + 1, 0), idx;
    for (int s = 0; s < S; ++s) {
      off[s] = (int)idx.size();
      for (int w = 0; w < (int)wallsHost_.size(); ++w)
        if (wallScene_[w] < 0 || wallScene_[w] == s)
          idx.push_back(w);
    }
    off[S] = (int)idx.size();
    sceneWallIdxD_.ensure(std::max<size_t>(idx.size(), 1), false, stream_);
    if (!idx.empty())
      cudaCheck(cudaMemcpyAsync(sceneWallIdxD_.p, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice, stream_), "H2D");
    cudaCheck(cudaMemcpyAsync(sceneWallOffD_.p, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice, stream_), "H2D");
    ensureContactCapacity();
    refreshDev();
    sync();
    sceneWallsDirty_ = false;
  }
  if (sceneParamsDirty_) {
    sceneMaxScale_.zero(stream_, S);
    if (numReal_ > 0)
      ++launches_, kSceneMaxScale<<<gridFor(numReal_), kBlock, 0, stream_>>>(d_, numReal_, sceneMaxScale_.p);
    KCHECK("scene max scale");
    std::vector<R> mx(S), par(3 * (size_t)S);
    cudaCheck(cudaMemcpyAsync(mx.data(), sceneMaxScale_.p, S * sizeof(R), cudaMemcpyDeviceToHost, stream_), "D2H");
    sync();
    for (int s = 0; s < S; ++s) {
      const bool empty = sceneFirstHost_[s + 1] == sceneFirstHost_[s];
      const R maxRad = empty ? gs_ * baseRadius_ : mx[s] * gs_ * baseRadius_;
      par[3 * s] = R(0.1) * maxRad;
      par[3 * s + 1] = sceneE_[s];
      par[3 * s + 2] = sceneMu_[s];
    }
    cudaCheck(cudaMemcpyAsync(sceneParams_.p, par.data(), par.size() * sizeof(R), cudaMemcpyHostToDevice, stream_), "H2D");
    sync();
    sceneParamsDirty_ = false;
  }
  ++launches_, kSceneBegin<<<gridFor(S), kBlock, 0, stream_>>>(scn_.p, S, sceneParams_.p);
  KCHECK("scene begin");
}
// after the manifold reduction: first pair / plane / wall contact and first manifold of every scene
template <class R>
void Sim<R>::batchBounds(int nm) {
  const int S = numScenes_;
  const int t0 = lastTot_[0], t1 = t0 + lastTot_[1], t2 = t1 + lastTot_[2];
  int* cf = sceneConFirstD_.p;
  ++launches_, kSceneBounds<<<gridFor(S + 1), kBlock, 0, stream_>>>(cab_.p, 0, t0, S, sceneFirstD_.p, cf);
  ++launches_, kSceneBounds<<<gridFor(S + 1), kBlock, 0, stream_>>>(cab_.p, t0, t1, S, sceneFirstD_.p, cf + (S + 1));
  ++launches_, kSceneBounds<<<gridFor(S + 1), kBlock, 0, stream_>>>(cab_.p, t1, t2, S, sceneFirstD_.p, cf + 2 * (S + 1));
  ++launches_, kSceneBounds<<<gridFor(S + 1), kBlock, 0, stream_>>>(mab_.p, 0, nm, S, sceneFirstD_.p, sceneManFirstD_.p);
  KCHECK("scene bounds");
}

template class Sim<float>;
template class Sim<double>;

}  // namespace pdem
