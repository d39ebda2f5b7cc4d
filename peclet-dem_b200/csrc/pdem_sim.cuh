// Host side of the B200 substep: the Simulation facade state (src/sim.hpp:909-1670) and the step
// orchestration (src/sim.hpp:97-488, 494-541, 628-750), owning all device memory.
#pragma once
#include <cstdlib>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <limits>
#include <map>
#include <memory>
#include <tuple>
#include <utility>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "pdem_common.cuh"

namespace pdem {
template <class R>
struct SolveP;  // pdem_solve.cuh


struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
void cudaCheck(cudaError_t e, const char* what);

// device allocations made by growable buffers since load (instrumentation)
extern long gDeviceAllocs;

// growable device buffer (contents not preserved unless asked), allocated in stream order from the
// device's default pool: growth neither waits for the device nor returns memory to the driver (the
// pool keeps freed blocks; its release threshold is raised when a simulation is created), so a
// scene whose contact count climbs while it settles reallocates without stalling its stream
template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() {
    if (p)
      cudaFree(p);  // the owner synchronised its stream; cudaFree accepts pool allocations
  }
  void ensure(size_t want, bool preserve = false, cudaStream_t s = 0) {
    if (want <= n && p)
      return;
    size_t cap = want < 1 ? 1 : want;
    if (p && cap < n + n / 2)
      cap = n + n / 2;  // grow geometrically: counts that creep up each substep reallocate rarely
    T* q = nullptr;
    ++gDeviceAllocs;
    cudaCheck(cudaMallocAsync(reinterpret_cast<void**>(&q), cap * sizeof(T), s), "cudaMallocAsync");
    cudaCheck(cudaMemsetAsync(q, 0, cap * sizeof(T), s), "cudaMemset");
    if (preserve && p && n)
      cudaCheck(cudaMemcpyAsync(q, p, n * sizeof(T), cudaMemcpyDeviceToDevice, s), "cudaMemcpy");
    if (p)
      cudaCheck(cudaFreeAsync(p, s), "cudaFreeAsync");  // after every use queued on s so far
    p = q;
    n = cap;
  }
  void zero(cudaStream_t s, size_t count = 0) {
    if (p)
      cudaCheck(cudaMemsetAsync(p, 0, (count ? count : n) * sizeof(T), s), "cudaMemset");
  }
};

struct XAdjAccess;  // the XPBD adjoint (pdem_xadj.cu) reads the step's buffers

template <class R>
class Sim {
  friend struct XAdjAccess;

 public:
  explicit Sim(int capacity);
  ~Sim();
  // the XPBD adjoint's record and workspace (pdem_xadj.cu), created by its first use
  std::shared_ptr<void> xadj_;

  // ---- facade (src/sim.hpp:943-1424) ----
  void initializeShape(int type, R radius, R height, R thick);
  void setShellPoints(const std::vector<R>& pts);
  void setSdfShape(const std::vector<R>& grid, int nx, int ny, int nz, const R* origin, const R* spacing,
                   const std::vector<R>& shell, const R* invI, R boundingRadius);
  void setDomain(R lx, R ly, R lz, bool px, bool py, bool pz);
  void setDomainMinMax(const R* mn, const R* mx);
  void enablePeriodicity(bool x, bool y, bool z);
  void setGravity(R gx, R gy, R gz) { g_[0] = gx, g_[1] = gy, g_[2] = gz; }
  void setThermostat(R T, R tau, R kB) { thT_ = T, thTau_ = tau, thKB_ = kB; }
  void setSolverIterations(int pos, int vel) { posIters_ = pos, velIters_ = vel; }
  void setVelocityUseGS(bool b) { useGS_ = b, topoValid_ = false; }
  void setStabilizationMode(const std::string& m);
  void setHertzMaterial(int mat, R E, R nu);
  void setGlobalScale(R s) { gs_ = s, skin_ = R(0.1) * s, vValid_ = false; }
  void setDt(R dt) { dt_ = dt; }
  void setMaterialParams(R en, R et, R mu) { eN_ = en, eT_ = et, mu_ = mu; }
  void setMaterialIds(const int* ids, int n);
  void setPairMaterial(int a, int b, R e, R mu);
  void setWallMaterialId(int wid, int mat);
  void addPlane(const R* p, const R* n);
  int addSdfWall(const std::vector<R>& grid, int nx, int ny, int nz, const R* origin, const R* spacing, R e,
                 R mu);
  void setWallVelocity(int idx, const R* lin, const R* ang, const R* center);
  void setPositions(const R* xyz, int n);
  void setRows(int field, const R* a, int n);  // velocities, forces, quats, angvel, invI, invMass
  void clearExternalForces();
  void setScales(const R* s, int n);
  void setScalesUniform(R s);
  void setGrowthParams(R rate, R nf);
  R growthFactor() const { return gf_; }
  R growthRate() const { return gr_; }
  void getRows(int field, R* out, long cap);  // positions .. masses
  void setRowsD(int field, const double* a, int n);  // fields 0-4 of setRows, packed on the device
  void getRowsD(int field, double* out, long cap);   // fields 0-4 of getRows, unpacked on the device
  void step(R dt);
  void stepHertz(R dt, int substeps, R skinFrac);
  R computeOverlaps();
  int numParticles() const { return numReal_; }
  int numContacts();
  int numManifolds();
  R maxOverlap();
  void sync();

  // ---- diagnostics (canonical order) ----
  void counts(long* out);
  long getPairs(int* out, long cap);
  long getContacts(double* out, long cap, bool muOnly);
  long getManifolds(double* out, long cap);
  long getColors(bool manifold, int* out, long cap);
  long getLambda(double* out, long cap);
  long getPairKeys(unsigned long long* out, long cap);
  long getLedger(unsigned long long* keys, double* vals, long cap);
  long getGrounded(int* out, long cap);
  long getPosLambda(double* out, long cap);
  long getHertz(unsigned long long* keys, double* xi, long cap);
  void setMaxContacts(int n);

  // host-side facade state
  int capacity_ = 0, numReal_ = 0, numParticles_ = 0, maxPairs_ = 0, maxContacts_ = 0;
  int shellPoints_ = 0;
  // bytes of the active shape's point shell that the shell narrowphase stages in shared memory
  // (0: too large, read from global memory)
  int shellStageBytes() const {
    const long b = (long)shellPoints_ * (long)sizeof(Q4<R>);
    return (shellPoints_ > 0 && b <= 32 * 1024) ? (int)b : 0;
  }
  R baseRadius_ = 1, defInvI_[3] = {R(2.5), R(2.5), R(2.5)};
  R dmin_[3] = {0, 0, 0}, dmax_[3] = {0, 0, 0}, dsize_[3] = {0, 0, 0};
  bool per_[3] = {false, false, false};
  R g_[3] = {0, 0, 0};
  R dt_ = R(1e-3), gs_ = 1, gr_ = 0, gf_ = -1, thT_ = 0, thTau_ = 0, thKB_ = 1;
  R eN_ = 0, eT_ = 0, mu_ = 0, skin_ = R(0.1), wallFrictionMax_ = 0;
  int posIters_ = 10, velIters_ = 0, stabMode_ = 1;
  bool useGS_ = true;
  int prevPairCount_ = 0;
  ShapeDesc<R> shape_{};
  std::vector<Q4<R>> shellHost_;
  std::vector<R> sdfGridHost_;
  std::vector<PlaneDesc<R>> planesHost_;
  std::vector<WallDesc<R>> wallsHost_;
  std::vector<R> wallGridHost_;
  std::vector<R> pairMatHost_;
  R hzE_[8], hzNu_[8];
  int hzNumPairs_ = -1, hzPrevCount_ = 0, hzNumWallCand_ = 0;
  R hzContactFrac_ = R(0.5);

  // ---- FP32-mixed form (meaningful for R = float): FP64 master positions / orientations ----
  void setMixed(bool on);
  void setMaster(int field, const double* a, int n);
  bool getMaster(int field, double* out, long cap);
  bool mixed_ = false;

  // ---- batched form: independent scenes in one body array, each stepped as it would be alone ----
  void setScenes(int S, const int* firstBody);
  void setSceneMaterial(int scene, R e, R mu);
  void setWallScene(int wall, int scene);
  long sceneCounters(double* out, long cap);
  int numScenes() const { return batch_ ? numScenes_ : 1; }

  cudaStream_t stream_ = nullptr;
  Dev<R> d_{};

  // ---- instrumentation: kernel launch count and opt-in per-stage device time ----
  enum Stage {
    ST_PREDICT, ST_GHOSTS, ST_BROAD, ST_NARROW, ST_MANIFOLD, ST_COLOR_V, ST_WARM, ST_VELOCITY, ST_STAB,
    ST_LEDGER, ST_FRICTION, ST_INTEGRATE, ST_COLOR_P, ST_POSITION, ST_COMMIT, ST_HERTZ_PAIRS, ST_HERTZ_REBUILD,
    ST_HERTZ_INTEGRATE, ST_END, ST_COUNT
  };
  long launches_ = 0;
  long sweeps_[4] = {0, 0, 0, 0};  // velocity, stabilization, position sweeps; substeps (profiled)
  long reuse_[3] = {0, 0, 0};      // substeps that kept: manifold grouping, contact colours, manifold colours
  bool prof_ = false;
  double stageMs_[ST_COUNT] = {};
  double stageHostMs_[ST_COUNT] = {};  // host wall time spent issuing each stage (launches, read-backs)
  long stageCalls_[ST_COUNT] = {};
  void profileEnable(bool on);
  // device-timeline interval between two calls (events on the library's stream; stop synchronises)
  void timerStart();
  double timerStop();
  cudaEvent_t tStart_ = nullptr, tStop_ = nullptr;
  void mark(int stage);
  void flushMarks();

 private:
  // device buffers
  DBuf<Q4<R>> pos_, vel_, angVel_, invI_, posPred_, velPred_, angVelPred_, quat_, quatPred_, extF_, dVel_,
      dAngVel_, dPos_;
  DBuf<R> invMass_, scale_, target_, rad_, planeFric_;
  DBuf<int> shapeId_, realIdx_, counts_;
  DBuf<uint8_t> grounded_, matId_;
  DBuf<long long> winner_;
  DBuf<u64> mask_;
  DBuf<int2> pairs_;
  DBuf<int2> cab_;
  DBuf<Q4<R>> cn_, crA_, crB_, cbv_;
  DBuf<int> cColor_, cSlot_;
  DBuf<R> posLamC_;
  DBuf<int2> mab_;
  DBuf<int> mnp_, mColor_;
  DBuf<Q4<R>> mN_, mTA_, mTB_, mrA_, mrB_, mwv_;
  DBuf<u64> pairKeys_, prevKeys_;
  DBuf<uint8_t> persistent_, sideFlags_;
  DBuf<int> heights_, ordChanged_, ordKeysIn_, ordKeys_, ordPermIn_, ordPerm_;  // "ordered" pass
  DBuf<R> sdfA_, sdfB_;  // get_sdf_grid ping-pong
  DBuf<int> colorListM_, colorListC_;  // colouring worklists (two halves each)
  DBuf<int> colorTail_;                // block list lengths and the tail's worklists
  DBuf<int> sdfState_;
  DBuf<R> lambda_, prevLambda_, vn0_, posImp_, prevPosImp_;
  DBuf<Q4<R>> lambdaT_, prevLambdaT_, vt0_;
  DBuf<ShapeDesc<R>> shapeD_;
  DBuf<Q4<R>> shellD_;
  DBuf<R> sdfGridD_;
  DBuf<PlaneDesc<R>> planesD_;
  DBuf<WallDesc<R>> wallsD_;
  DBuf<R> wallGridD_, pairMatD_, hzED_, hzNuD_;
  DBuf<Counters<R>> ctr_;
  int numSMs_ = 148;
  // batched form
  bool batch_ = false, sceneParamsDirty_ = true, sceneWallsDirty_ = true;
  bool maxScaleValid_ = false;  // maxScaleHost_ holds the largest scale of the real bodies
  // broadphase tree reuse: topology rebuilt when the body set changes or every kBvhRebuild substeps
  static constexpr int kBvhRebuild = 16;
  bool bvhValid_ = false;
  int bvhN_ = 0, bvhReal_ = 0, bvhAge_ = 0;
  // Verlet candidate superset (skin = half the contact margin): the step's pairs are filtered from it
  // topology reuse (contact list / manifold list equal to the previous substep's)
  DBuf<int2> prevCab_;
  DBuf<int4> prevMsig_;
  DBuf<int> topoFlags_;  // [0] the contact list differs, [1] the manifold list differs
  int prevNc_ = -1, prevNb_ = -1, prevNcM_ = -1, prevNm_ = 0, prevNmSig_ = -1, topoChecks_ = 0;
  int incKind_ = -1, incNe_ = -1;  // what the incidence buffers hold
  bool topoValid_ = false, lastSame_ = false, keptM_ = false, keptC_ = false;
  bool verlet_ = true, vValid_ = false;
  int vN_ = 0, vReal_ = 0, vCount_ = 0;
  R vMargin_ = R(0);
  DBuf<int2> vpairs_;
  DBuf<Q4<R>> vRef_;
  DBuf<int> vRefReal_, vKeep_, vOff_;
  R maxScaleHost_ = R(0);
  int numScenes_ = 1, maxSceneBodies_ = 0;
  std::vector<int> sceneFirstHost_;   // [S + 1] first body of each scene
  std::vector<R> sceneE_, sceneMu_;   // per-scene restitution and friction
  std::vector<int> wallScene_;        // per wall: its scene, or -1 for every scene
  DBuf<int> sceneOf_, sceneFirstD_, sceneWallOffD_, sceneWallIdxD_, sceneManFirstD_, sceneConFirstD_,
      sceneLeafFirstD_, bvhFirst_, bvhLast_;
  DBuf<SceneCtl<R>> scn_;
  DBuf<Q4<double>> posD_, quatD_;  // FP32-mixed form: master positions and orientations
  DBuf<double> rowStage_;           // host rows staged on the device (set/get of 4-wide fields)
  DBuf<R> sceneParams_, sceneMaxScale_;
  DBuf<int> sceneLpt_;  // scenes by decreasing body count: dispatch order of the per-scene loops
  DBuf<int> rankBad_;   // the contact rank scatter's rejection flag
  DBuf<int> colorHist_;  // the colouring launch's per-block colour histograms (both graphs)
  DBuf<int> ledFlag_, ledPos_;  // ledger order: in-order (or live) flags and their scan
  DBuf<int> ledGhost_, ledGPos_;    // ledger order with ghost images: ghost-manifold flags, scan
  DBuf<u64> ledOKeys_, ledOKeysS_;  // the ghost manifolds' keys
  DBuf<int> ledOIdx_, ledOIdxS_;    // and indices, before and after their sort
  bool ledgerSplit_ = false;        // this substep's ledger order merges the sorted ghost manifolds
  int ledgerGhosts_ = 0;            // their count (read back with the stabilization decision)
 public:
  long rankStats_[2] = {0, 0};  // substeps whose contact grouping was ranked, and ranked then rejected
 private:
  int lastTot_[3] = {0, 0, 0};
  Counters<R> detectCounters_{};  // host copy of the counters after the narrowphase (H2D source)
  void batchBegin();
  long wallsPerBody() const;
  void batchBounds(int nm);
  void ctl(int op, R thr, int mode);
  DBuf<unsigned> gbar_;        // grid barrier of the persistent loops
  DBuf<long long> winner2_;    // second winner array of the colouring rounds
  DBuf<long long> winnerP_, winnerP2_;  // winner arrays of the contact colouring
  DBuf<u64> maskP_;                     // colour masks of the contact colouring
  DBuf<int> colorAux_;         // colouring, per graph (5 each): remaining counts [3], statistics [2]
  // scratch
  DBuf<char> cubTmp_;
  DBuf<int> iA_, iB_, iC_, iD_, iE_;
  DBuf<u64> kA_, kB_;
  DBuf<unsigned> uA_, uB_;
  DBuf<R> rA_, rB2_;
  DBuf<Q4<R>> qA_, qB_, qC_;
  static constexpr int kGroundRing = 32;  // 255 / 8 < 32 substeps of decay erase any level
  DBuf<int4> gRing_[kGroundRing];
  int gRingNm_[kGroundRing] = {}, gRingReal_[kGroundRing] = {};
  int gRingScenes_[kGroundRing] = {};   // batched form: scenes of the slot (0: one scene)
  DBuf<int> gRingScn_[kGroundRing];     // batched form: first manifold of each scene in the slot
  long gLog_ = 0, gCheckpoint_ = 0;
  DBuf<int> gscratch_;
  DBuf<double> thermo_;
  // broadphase scratch
  DBuf<char> bvhBoxes_, bvhNodes_;
  DBuf<u64> codes_, codesAlt_, bounds_;
  DBuf<u64> radixK_;            // the Morton sort's scratch (pdem_radix.cuh)
  DBuf<int> radixV_, radixH_;
  DBuf<int> bidx_, bidxAlt_, left_, right_, parent_, flag_, qcnt_, qoff_, rowCnt_, bflag_;
  DBuf<int2> slots_;
  // manifold reduction scratch (kept for the position-impulse commit)
  DBuf<u64> ckeys_, ckeysS_;
  DBuf<int> cperm_, cpermIn_, head_, headScan_, segStart_;
  // colour orders
  DBuf<int> mOrder_, mOff_, cOrder_, cOff_;
  // ledger sort
  DBuf<u64> lkeysS_, lkeysIn_;
  DBuf<int> lperm_, lpermIn_;
  // incidence lists
  DBuf<int> incKeys_, incKeysS_, incVals_, incValsS_, incOff_;
  // Hertz
  DBuf<Q4<R>> hzXi_, hzPrevXi_, hzXiWall_, hzRefPos_;
  DBuf<u64> hzKeys_, hzPrevKeys_;
  DBuf<R> hzSnPair_, hzSnWall_;
  DBuf<int> hzWallCand_, hzCandOff_, hzOnW_;
  DBuf<Q4<R>> hzFW_, hzTW_;
  struct Mark {
    int stage;
    cudaEvent_t ev;
    double host;  // host steady-clock seconds when the stage's first launch was being issued
  };
  std::vector<Mark> marks_;
  std::vector<cudaEvent_t> evFree_;

  void allocate(int cap, int maxPairs, int maxContacts);
  void allocContactBuffers(int mc);
  void ensureCapacity(int nc);
  void ensureContactCapacity();
  void refreshDev();
  void uploadShape();
  void uploadWalls();
  void uploadHertzMaterials();
  int ghostCapacity(int nReal, R band) const;
  R maxOwnedRadius();
  void resetGhosts(R band);
  int findCollisionsGrow(R margin, const Q4<R>* P);
  int findCollisions(R margin, int cap, int2* out, R extra = R(0));
  int findCollisionsVerlet(R margin);
  void detectAll(R margin);
  int reduceManifolds(int nc);
  void colorBoth(int nm, int nc, int& ncolV, int& velLeft, int& ncolP, int& posLeft);
  void colorOrder(bool manifold, int ne, int ncol);
  void buildIncidence(int kind, int ne, int nb);
  void logSupportGraph(int nm, V3<R> gHat);
  void ensureGrounded();
  void demStep();
  Counters<R> readCounters();
  // small read-backs: device -> a pinned block, queued without a host wait (a copy into pageable
  // memory waits for its own completion, so a group of them cost a round trip each); sync() then
  // copies each value to its host destination. Destinations must live until that sync().
  void readBack(void* host, const void* dev, size_t bytes);
  struct PendingRead {
    void* host;
    size_t off, bytes;
  };
  std::vector<PendingRead> pending_;
  char* pin_ = nullptr;
  size_t pinOff_ = 0;
  static constexpr size_t kPinBytes = 1 << 16;
 public:
  void dropPending() {  // after an exception between a read-back and its sync
    pending_.clear();
    pinOff_ = 0;
  }
 private:
  template <class K>
  int coopGrid(K kernel, int block);
  template <class K, class... A>
  void launchCoopB(K kernel, int block, A... args);
  template <class K, class... A>
  void launchCoop(K kernel, A... args);
  // cooperative launch with `smem` bytes of dynamic shared memory (resident blocks counted with it)
  template <class K, class... A>
  void launchCoopSmem(K kernel, int block, size_t smem, A... args);
  std::map<std::tuple<const void*, int, size_t>, int> coopPerSmem_;  // by (kernel, block, smem)
  // one thread-block cluster of sweepClusterBlocks_ blocks; false when such a cluster cannot be
  // resident
  template <class K, class... A>
  bool launchCluster(K kernel, A... args);
  // one cluster of `blocks` blocks of `block` threads with `smem` bytes of dynamic shared memory;
  // false (nothing launched) when such a cluster cannot be resident. Residency is cached per kernel.
  template <class K, class... A>
  bool launchClusterCfg(K kernel, int blocks, int block, size_t smem, A... args);
  // largest colouring (entries of the larger graph) run in one cluster (PDEM_COLOR_CLUSTER_ENTRIES)
  long colorClusterEntries_ = [] {
    const char* e = std::getenv("PDEM_COLOR_CLUSTER_ENTRIES");
    return e ? std::max(0L, std::strtol(e, nullptr, 10)) : 32768L;
  }();
  std::map<const void*, int> clusterOk_;  // per kernel: 1 resident, 0 not
  // velocity-sweep records of the one-cluster loops (kPackPgs), packed once per substep
  PgsRecs<R> packPgs(int nm, int ncol);
  DBuf<Q4<R>> pgsQ_;
  DBuf<int4> pgsIds_;
  long pgsCap_ = 0;
  long substepId_ = 0, pgsPackedAt_ = -1;
  // blocks of the one-cluster sweep loop (PDEM_SWEEP_CLUSTER: 8, the portable size, or 16, which
  // needs the non-portable cluster attribute) and the largest entry list it takes
  // (PDEM_SWEEP_CLUSTER_ENTRIES); larger lists sweep on the cooperative grid
  int sweepClusterBlocks_ = [] {
    const char* e = std::getenv("PDEM_SWEEP_CLUSTER");
    const long v = e ? std::strtol(e, nullptr, 10) : 16;
    return v == 8 ? 8 : 16;
  }();
  long sweepClusterEntries_ = [] {
    const char* e = std::getenv("PDEM_SWEEP_CLUSTER_ENTRIES");
    // default: up to 8 entries a thread of 16 x 256 (about one entry a thread per colour step at
    // the 8-12 colours of a settled pile). Measured on the 4,096-sphere settled bed (12.4k
    // manifolds): the velocity loop 0.57 ms per substep on the cooperative grid, 0.47 in one cluster
    return e ? std::max(0L, std::strtol(e, nullptr, 10)) : 32768L;
  }();
  std::map<std::pair<const void*, int>, int> coopPer_;  // resident blocks per SM, by (kernel, block)
  template <class T>
  void sortPairs(const T* kin, T* kout, const int* vin, int* vout, int n, int endBit);
  void orderedStabilization(int nm, V3<R> gHat, const SolveP<R>& ss, R vRestS);
  // the multilevel stabilization pass and its buffers (pdem_multilevel.cuh)
  void multilevelStabilization(int nm, int ncol, const SolveP<R>& ss, R vRestS, R gMag);
  DBuf<long long> mlPacked_, mlWin_;
  DBuf<int> mlParent_, mlGrp_, mlMate_, mlFlag_, mlPos_, mlInt_;
  DBuf<u64> mlMask_;
  DBuf<R> mlMassG_, mlInvMassG_, mlQS_;
  DBuf<Q4<R>> mlVelG_, mlVelG0_;
 public:
  // launch shape autotuner of the per-scene sweep loops: the chosen block (0 while tuning) and the
  // mean sweep-loop time of each candidate (ms per substep)
  int tunedSceneBlock() const { return tuning_ ? 0 : sceneBlock_; }
  const float* tuneMs() const { return tuneMs_; }
  static constexpr int kTuneCands = 4, kTuneRounds = 3;
  static constexpr int kTuneBlocks[kTuneCands] = {64, 128, 256, 512};
 private:
  int sceneBlock() const;
  void tuneBegin();
  void tuneEnd();
  int sceneBlock_ = 128, tuneStep_ = 0;
  bool tuning_ = false, tuneOpen_ = false;
  cudaEvent_t tuneEv_[kTuneCands * kTuneRounds][2] = {};
  float tuneMs_[kTuneCands] = {0, 0, 0, 0};
 public:
  // zero-copy device arrays (get_*_view): 0 positions, 1 velocities, 2 external forces (rows of 4,
  // the first 3 used), 3 inverse mass (rows of 1); synchronises the stream first
  void deviceView(int field, void** ptr, long* rows, int* rowStride) {
    if (field < 0 || field > 3)
      throw std::invalid_argument("device view: field must be 0..3");
    sync();
    *rows = numReal_;
    *rowStride = field == 3 ? 1 : 4;
    *ptr = field == 0 ? (void*)pos_.p : field == 1 ? (void*)vel_.p : field == 2 ? (void*)extF_.p : (void*)invMass_.p;
  }
  std::vector<R> sdfGrid(int rx, int ry, int rz);  // get_sdf_grid, flat x-fastest
  void lastCounters(long* sizes, int* ints, double* maxOverlap);
 private:
  int ncolVLast_ = 0, ncolPLast_ = 0;  // colours of the last substep's two colourings
  int colorRounds_[2] = {0, 0};         // Jones-Plassmann rounds of the last manifold / contact colouring
  // block size of the colouring launch (PDEM_COLOR_BLOCK fixes it: 256, 512 or 1024). In the
  // batched form, without the variable, it is tuned online: the first kColorTuneCands x
  // kTuneRounds colourings cycle through the candidates, timed with events, and the fastest stays
  // (the colours do not depend on it: the rounds' winners are maxima of keys)
  int colorBlock_ = [] {
    const char* e = std::getenv("PDEM_COLOR_BLOCK");
    const int b = e ? (int)std::strtol(e, nullptr, 10) : 1024;
    return (b == 256 || b == 512) ? b : 1024;
  }();
  bool colorTuning_ = std::getenv("PDEM_COLOR_BLOCK") == nullptr;
  int colorTuneStep_ = 0;
  cudaEvent_t colorTuneEv_[3 * 3][2] = {};
  float colorTuneMs_[3] = {0, 0, 0};
 public:
  static constexpr int kColorTuneCands = 3;
  static constexpr int kColorTuneBlocks[kColorTuneCands] = {256, 512, 1024};
  // the colouring block the batched form's autotuner chose (0 while tuning) and each candidate's
  // mean colouring-launch time (ms)
  int tunedColorBlock() const { return (batch_ && colorTuning_) ? 0 : colorBlock_; }
  const float* colorTuneMs() const { return colorTuneMs_; }
 private:
  // entries left (both colourings) at which block 0 alone finishes the colouring; PDEM_COLOR_TAIL
  // overrides it (0 .. kColorTailMax). Measured: 1024 and 4096 alike on the 262k-sphere step, 1024
  // 6 % faster on the batched drums, 16384 and up far slower (one block, many entries a round)
  int colorTailAt_ = [] {
    const char* e = std::getenv("PDEM_COLOR_TAIL");
    const long v = e ? std::strtol(e, nullptr, 10) : 1024;
    return (int)std::max(0L, std::min(v, 1L << 30));  // capped at kColorTailMax where used
  }();
  // back-off (ns) between polls of a waiting block at a grid barrier; PDEM_BARRIER_SLEEP_NS
  // overrides it
  // polls before a grid-barrier wait gives up (setBarrierSpins; <= 0 restores kBarrierSpins)
  long barrierSpins_ = kBarrierSpins;
 public:
  void setBarrierSpins(long n) { barrierSpins_ = n > 0 ? n : kBarrierSpins; }
 private:
  void clearLoopError();
  unsigned barrierSleepNs_ = [] {
    const char* e = std::getenv("PDEM_BARRIER_SLEEP_NS");
    return e ? (unsigned)std::strtoul(e, nullptr, 10) : 64u;
  }();
  template <class T>
  void exclusiveSum(const T* in, T* out, int n);
  template <class T>
  void inclusiveSum(const T* in, T* out, int n);
  // Hertz engine
  void hertzCommitHistory();
  void hertzRebuildPairs(R skin);
  int hertzWallCandidates(R skin);
};

}  // namespace pdem
