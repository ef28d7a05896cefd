// tl_system.cu -- host side of the B200 tet FEM step: device memory of a
// resident system, the step's control flow (generalized-alpha substeps, the
// 3-read elastic path and the plastic Newton path of talus::deformable::step,
// solver.cc:3472-4369, 5829-5900) over the kernels of tl_kernels.cuh, and the
// C ABI of include/talus_fem.h.

#include "../../include/talus_fem.h"
#include "tl_kernels.cuh"
#include "tl_adjoint.cuh"
#include "tl_floating.cuh"
#include "tl_sell.cuh"
#include "tl_sell_build.h"
#include "tl_factor.cuh"
#include "tl_factor_host.h"
#include "tl_validate.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <type_traits>
#include <thread>
#include <vector>

#include <unistd.h>

using namespace tl;

namespace {

struct CudaError {
  cudaError_t code;
  const char* what;
};

#define TL_CUDA(call)                                  \
  do {                                                 \
    const cudaError_t e_ = (call);                     \
    if (e_ != cudaSuccess) throw CudaError{e_, #call}; \
  } while (0)

struct StatusError {
  int32_t status;
  std::string what;
};

template <class T>
struct DevBuf {
  T* ptr = nullptr;
  size_t count = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() {
    if (ptr) cudaFree(ptr);
  }
  void alloc(size_t n) {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    count = n;
    if (n) TL_CUDA(cudaMalloc(&ptr, n * sizeof(T)));
  }
  void zero(cudaStream_t s) {
    if (count) TL_CUDA(cudaMemsetAsync(ptr, 0, count * sizeof(T), s));
  }
  void upload(const T* host, size_t n, cudaStream_t s, size_t offset = 0) {
    if (n) TL_CUDA(cudaMemcpyAsync(ptr + offset, host, n * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void download(T* host, size_t n, cudaStream_t s, size_t offset = 0) const {
    if (n) TL_CUDA(cudaMemcpyAsync(host, ptr + offset, n * sizeof(T), cudaMemcpyDeviceToHost, s));
  }
};

template <class T>
struct PinnedBuf {
  T* ptr = nullptr;
  size_t count = 0;
  ~PinnedBuf() {
    if (ptr) cudaFreeHost(ptr);
  }
  T* get(size_t n) {
    if (n > count) {
      if (ptr) cudaFreeHost(ptr);
      ptr = nullptr;
      TL_CUDA(cudaMallocHost(&ptr, n * sizeof(T)));
      count = n;
    }
    return ptr;
  }
};

uint32_t tilesOf(uint64_t n) { return uint32_t((n + TILE - 1) / TILE); }

// Generalized-alpha rule (solver.cc:531-566) in double.
struct Rule {
  double alphaMass, alphaForce, beta, gamma;
};
Rule ruleOf(double spectral) {
  const double held = std::clamp(spectral, 0.0, 1.0);
  Rule r;
  r.alphaMass = (2.0 * held - 1.0) / (held + 1.0);
  r.alphaForce = held / (held + 1.0);
  r.gamma = 0.5 - r.alphaMass + r.alphaForce;
  r.beta = 0.25 * (1.0 - r.alphaMass + r.alphaForce) * (1.0 - r.alphaMass + r.alphaForce);
  return r;
}

constexpr uint32_t ANCHORED_READS = 3u;       // solver.cc:11
constexpr uint32_t INVERTED_SUBSTEPS = 4u;    // solver.cc:13
constexpr double LOADING_MARGIN = 1.0e-3;     // solver.cc:372
constexpr double PLASTIC_REDUCTION = 1.0e-2;  // solver.cc:374
constexpr double PLASTIC_RESOLUTION = 8.0;    // solver.cc:380
constexpr double FLOATING_TOLERANCE = 1.0e-5; // solver.cc:9

// Worker threads for the host side of state transfers, started on first use
// and kept until the process exits (up to 15 workers beside the calling
// thread; the pool is never destroyed, so no worker is joined at exit).  One
// job at a time: a job is a range split into contiguous parts, part 0 run by
// the caller.
class HostPool {
 public:
  static HostPool& instance() {
    static HostPool* pool = new HostPool();
    return *pool;
  }
  // Workers usable from this process: none in a child forked after the pool
  // started (its threads were not copied).
  size_t workers() const { return getpid() == owner_ ? threads_.size() : 0; }
  // Runs body(part) for part in [0, parts), parts <= workers() + 1.
  void run(size_t parts, const std::function<void(size_t)>& body) {
    std::lock_guard<std::mutex> call(callMutex_);
    {
      std::lock_guard<std::mutex> lk(m_);
      job_ = &body;
      parts_ = parts;
      next_ = 1;
      pending_ = parts - 1;
      ++generation_;
    }
    cv_.notify_all();
    body(0);
    std::unique_lock<std::mutex> lk(m_);
    done_.wait(lk, [&] { return pending_ == 0; });
    job_ = nullptr;
  }

 private:
  HostPool() : owner_(getpid()) {
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    for (unsigned i = 1; i < hw; ++i) threads_.emplace_back([this] { loop(); });
  }
  void loop() {
    uint64_t seen = 0;
    for (;;) {
      std::unique_lock<std::mutex> lk(m_);
      cv_.wait(lk, [&] { return generation_ != seen && next_ < parts_; });
      seen = generation_;
      while (next_ < parts_) {
        const size_t part = next_++;
        const std::function<void(size_t)>* job = job_;
        lk.unlock();
        (*job)(part);
        lk.lock();
        if (--pending_ == 0) done_.notify_one();
      }
    }
  }
  std::vector<std::thread> threads_;
  std::mutex m_, callMutex_;
  std::condition_variable cv_, done_;
  const std::function<void(size_t)>* job_ = nullptr;
  size_t parts_ = 0, next_ = 0, pending_ = 0;
  uint64_t generation_ = 0;
  pid_t owner_;
};

// Host loops over [0, n) split across the pool (state conversion of large
// bodies); small ranges run inline.  The body must not throw.
template <class F>
void parallelFor(size_t n, F&& body) {
  if (n < (size_t(1) << 16)) {
    body(size_t(0), n);
    return;
  }
  HostPool& pool = HostPool::instance();
  const size_t parts = std::min<size_t>(pool.workers() + 1, n >> 14);
  if (parts <= 1) {
    body(size_t(0), n);
    return;
  }
  const size_t per = (n + parts - 1) / parts;
  const std::function<void(size_t)> job = [&](size_t p) { body(p * per, std::min(n, (p + 1) * per)); };
  pool.run(parts, job);
}

// Whether p is page-locked host memory (tl_host_register, cudaHostAlloc).
bool pinnedHost(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

// memcpy split across the pool.
void parallelCopy(void* dst, const void* src, size_t bytes) {
  parallelFor(bytes, [&](size_t b0, size_t b1) {
    std::memcpy(static_cast<unsigned char*>(dst) + b0, static_cast<const unsigned char*>(src) + b0, b1 - b0);
  });
}


struct HostBody {
  uint32_t nodes = 0, tets = 0;
  uint32_t laneBase = 0, lanes = 0;  // the body's material lanes in the system's lane table
  bool anyAnchored = false, anyYields = false;
  std::vector<double> rest;  // [3 V] for position <-> displacement
  double restCentre[3] = {0.0, 0.0, 0.0};  // mass-weighted rest centre (of the stored rest positions)
  double mass = 0.0;
  // floats (solver.cc:2964-2971): no anchored node and the rigid split on
  bool floats(uint32_t split) const { return split != TL_RIGID_SPLIT_OFF && !anyAnchored; }
};

}  // namespace

struct tl_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int sms = 0;
  std::string last_error;
};

struct RolloutBase {
  virtual ~RolloutBase() = default;
  virtual void forward(tl_step_report* report, double* seconds) = 0;
  virtual void adjoint(const double* dxT, const double* dvT, double* dE, double* dv0, double* dx0,
                       double* seconds) = 0;
};

struct SystemBase {
  virtual ~SystemBase() = default;
  virtual void setYoungs(uint32_t body, const double* youngs) = 0;
  virtual void evaluate(uint32_t body, const tl_settings& settings, double* forces, uint8_t* yielding) = 0;
  virtual std::unique_ptr<RolloutBase> rollout(const tl_rollout_desc& desc, const tl_settings& settings) = 0;
  virtual void stateSet(uint32_t body, int32_t dtype, const void* x, const void* v, const void* a, const void* rot,
                        const void* plastic) = 0;
  virtual void stateGet(uint32_t body, int32_t dtype, void* x, void* v, void* a, void* rot, void* plastic) = 0;
  virtual int32_t step(const tl_settings& set, const double g[3], double dt, tl_step_report* reports) = 0;
  virtual void tune(uint32_t blocksPerSm, uint32_t graph) = 0;
  virtual void tuneShape(uint32_t knob, uint32_t value) = 0;
  virtual void setSolver(uint32_t form) = 0;
  virtual void useFactor(uint32_t enable, uint32_t budget) = 0;
  virtual void factorStats(tl_factor_stats* out) = 0;
  virtual void setPlasticity(uint32_t mode) = 0;
  virtual void expireWait(int32_t solve) = 0;
  virtual bool plasticUsed(uint32_t law) const = 0;
  virtual void setFlowLimits(uint32_t body, uint32_t lane, double crushStress, double crushLimit,
                             double plasticMax) = 0;
  std::vector<uint32_t> trace;  // TL_FLAG_TRACE: iterations of each PCG launch (body 0)
  // the last step's per-substep records of every body ([bodies][SUBSTEP_RECORDS]) and substep counts
  std::vector<SubstepRecordDev> substepRecords;
  std::vector<uint32_t> substepCounts;
  uint32_t bodies = 0;
  uint64_t nodes = 0, tets = 0;
};

// The destroy calls use only `device`, so handles may be destroyed in any
// order (a garbage collector does not keep creation order).
struct tl_system {
  tl_ctx* ctx = nullptr;
  int device = 0;
  std::unique_ptr<SystemBase> impl;
};

struct tl_rollout {
  tl_system* system = nullptr;
  int device = 0;
  std::unique_ptr<RolloutBase> impl;
};

namespace {

// One block at the persistent kernels' grid barrier with one barrier already
// counted: the goal (two arrivals) needs an arrival that never comes, so the
// bounded wait runs out and records TL_ERR_TIMEOUT.
// A node array of the caller's layout ([3 count] of H) into the state
// (displacement u = x - X when rest is given), in FP64 as the host
// conversion does it, so both give the same bits.
template <class S, class H>
__global__ void __launch_bounds__(TILE) kNodeStateIn(Vec4<S>* dst, const H* src, const double* rest, uint32_t count) {
  const uint32_t n = blockIdx.x * TILE + threadIdx.x;
  if (n >= count) return;
  double x = double(src[3 * size_t(n)]), y = double(src[3 * size_t(n) + 1]), z = double(src[3 * size_t(n) + 2]);
  if (rest) {
    x -= rest[3 * size_t(n)];
    y -= rest[3 * size_t(n) + 1];
    z -= rest[3 * size_t(n) + 2];
  }
  dst[n] = Vec4<S>{S(x), S(y), S(z), S(0)};
}
// And back (x = X + u when rest is given).
template <class S, class H>
__global__ void __launch_bounds__(TILE) kNodeStateOut(H* dst, const Vec4<S>* src, const double* rest, uint32_t count) {
  const uint32_t n = blockIdx.x * TILE + threadIdx.x;
  if (n >= count) return;
  const Vec4<S> v = src[n];
  double x = double(v.x), y = double(v.y), z = double(v.z);
  if (rest) {
    x += rest[3 * size_t(n)];
    y += rest[3 * size_t(n) + 1];
    z += rest[3 * size_t(n) + 2];
  }
  dst[3 * size_t(n)] = H(x);
  dst[3 * size_t(n) + 1] = H(y);
  dst[3 * size_t(n) + 2] = H(z);
}

__global__ void __launch_bounds__(TILE) kWaitLimitCheck(GridSyncDev* sync) {
  unsigned int k = 1;
  (void)countBarrier(sync, k);
}

template <class S> struct Rollout;

template <class S>
struct System final : SystemBase {
  tl_ctx* ctx;
  cudaStream_t st;
  uint32_t B = 0, Vp = 0, Tp = 0, nodeTiles = 0, elemTiles = 0;
  std::vector<HostBody> hb;
  std::vector<BodyDev> bodyHost;
  uint32_t launches = 0;
  // device buffers
  DevBuf<BodyDev> dBody;
  DevBuf<BodyStepDev> dStep;
  DevBuf<MatDev> dMat;
  DevBuf<double> dFlim;          // [3 lanes] crush stress, crush limit, plastic cap (finite-strain flow)
  std::vector<double> hFlim;
  DevBuf<uint32_t> dNodeTileBody, dElemTileBody;
  DevBuf<Vec4<S>> rest4, pres, u, v, a, carried, shifted, weighted, total, incr, lowest, right, pre0, pre1, r, z, p, ap, w;
  DevBuf<uint8_t> anch;
  DevBuf<uint32_t> start, entry, lane;
  DevBuf<uint4> tet;
  DevBuf<double> dm, vold, eyoung;
  DevBuf<S> dms, vols, op, de2;
  DevBuf<Vec4<S>> plast, fe, de, ye, onorm;
  DevBuf<OpRec<S>> orec;
  // two-level assembly structures (single-body PCG)
  DevBuf<uint2> tileMeta;
  DevBuf<uint16_t> tileOff, tileEnt;
  DevBuf<Vec4<S>> slotPart;
  DevBuf<uint32_t> nsStart, nsSlot;
  DevBuf<uint4> nsInline;
  DevBuf<uint32_t> tileNode;
  DevBuf<uint2> eloc;
  DevBuf<double> blkPart;
  // assembled block matrix of the single-body PCG (tl_sell.cuh)
  bool sellReady = false;
  uint32_t sellRows = 0, sellSlices = 0, sellPositions = 0, sellStride = 0;
  int sellPerSm = 0, batchSellPerSm = 0, batchPipePerSm = 0;
  uint32_t elementGrid[3] = {0, 0, 0};  // resident element-pass grids: corotated, SNH, Hencky rest
  // launch shapes of the assembled PCG (tl_system_tune_shape): column slots per round trip of a
  // matrix row (0: the kernel's default) and resident blocks per SM of the batched kernels (0: 4)
  uint32_t tuneRowGroup = 0, tuneBatchBlocks = 0;
  int sellPerSmOf[2] = {0, 0};  // kPcgSell with row groups 2 and 4
  uint32_t sellU() const { return tuneRowGroup ? tuneRowGroup : sellRowGroup<S>(); }
  uint32_t batchU() const { return tuneRowGroup ? tuneRowGroup : BATCH_ROW_GROUP; }
  int batchBlocks() const { return tuneBatchBlocks ? int(tuneBatchBlocks) : BATCH_BLOCKS; }
  const void* sellKernel() const {
    return sellU() == 2u ? (const void*)kPcgSell<S, 2> : (const void*)kPcgSell<S, 4>;
  }
  const void* batchKernel(bool twoPhase) const {
    const bool u4 = batchU() == 4u, b3 = batchBlocks() == 3;
    if (twoPhase)
      return u4 ? (b3 ? (const void*)kPcgBatchSell<S, 4, 3> : (const void*)kPcgBatchSell<S, 4, 4>)
                : (b3 ? (const void*)kPcgBatchSell<S, 2, 3> : (const void*)kPcgBatchSell<S, 2, 4>);
    return u4 ? (b3 ? (const void*)kPcgBatchSellPipe<S, 4, 3> : (const void*)kPcgBatchSellPipe<S, 4, 4>)
              : (b3 ? (const void*)kPcgBatchSellPipe<S, 2, 3> : (const void*)kPcgBatchSellPipe<S, 2, 4>);
  }
  int occupancyOf(const void* fn, size_t smem) const {
    int perSm = 0;
    TL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, fn, TILE, smem));
    return perSm;
  }
  DevBuf<Vec4<S>> sellP2;  // kPcgBatchSell's second search-direction buffer; z of kPcgBatchSellPipe
  DevBuf<Vec4<double>> pipeState;  // kPcgBatchSellPipe's FP64 recurrences [8][Vp], allocated at its first use
  DevBuf<uint32_t> sellSliceStart, sellGroupSlice, sellCol, sellCentry, sellDiag;
  DevBuf<uint4> sellUrec;  // kSellAssemble's per-block records
  uint32_t sellUpperCount = 0, sellColCache = 0;
  static constexpr uint32_t SELL_COL_CACHE_MAX = 32;  // column slots per thread in kPcgSell's shared memory
  static constexpr uint32_t SELL_AUTO_MIN_TETS = 32768;  // TL_SOLVER_AUTO: smallest body that is assembled
  DevBuf<S> sellVal;
  DevBuf<Vec4<S>> sellVec;
  int pcg1PerSm[2][2] = {{0, 0}, {0, 0}};   // resident blocks per SM, [law][tangent]
  int batchPerSm[2][2] = {{0, 0}, {0, 0}};
  int pcg1DampPerSm[2] = {0, 0};             // corotated law with stiffness damping, [tangent]
  int batchDampPerSm[2] = {0, 0};
  uint32_t tuneBlocksPerSm = 0;              // tl_system_tune: cap on the persistent grid (0 = occupancy)
  bool tuneGraph = true;                     // tl_system_tune: capture batched elastic steps in a CUDA graph
  uint32_t solverForm = TL_SOLVER_AUTO;      // tl_system_set_solver
  int gridOf(int perSm) const {
    const int use = tuneBlocksPerSm ? std::min<int>(perSm, int(tuneBlocksPerSm)) : perSm;
    return std::max(1, std::min(use * ctx->sms, int(std::max(nodeTiles, elemTiles))));
  }
  DevBuf<double> part, npart, epart;
  DevBuf<uint32_t> loading, yielding, counter;
  DevBuf<BodyAccDev> acc;
  DevBuf<CgBodyDev> cg;
  DevBuf<CgReportDev> cgrep;
  DevBuf<GridSyncDev> sync;
  // batched plastic Newton: per-body gate words and the bit the next launches test (0: no gate)
  DevBuf<uint32_t> gate;
  PinnedBuf<uint32_t> hGate;
  uint32_t gateBit = 0;
  DevBuf<SubstepRecordDev> subrec;   // [B][SUBSTEP_RECORDS] per-substep solve records of the current step
  PinnedBuf<SubstepRecordDev> hSubrec;
  void recordSubstep(uint32_t pass) {
    kSubstepRecord<S><<<(B + 255) / 256, 256, 0, st>>>(view(), subrec.ptr, pass);
    check();
  }
  // Keeps the downloaded records (hSubrec) and each body's substep count.
  void keepSubsteps(const uint32_t* substeps) {
    substepRecords.assign(hSubrec.ptr, hSubrec.ptr + size_t(B) * SUBSTEP_RECORDS);
    substepCounts.assign(substeps, substeps + B);
  }
  bool hasEyoung = false;
  bool hasDamping = false;   // some element's lane has stiffness damping
  bool hencky = false;       // TL_PLASTICITY_HENCKY: finite-strain flow from a per-tet plastic rest
  DevBuf<double> hk;         // [10][Tp] plastic map P (row-major planes), hardening variable
  bool evaluating = false;   // tl_evaluate: element forces only, no damping terms
  DevBuf<S> dtau, dfit;
  // floating bodies: the frame of each body, moment partials, frame velocities
  // and drives; allocated by the first step that has a floating body
  DevBuf<FrameDev> dFrame;
  DevBuf<double> fpart;
  DevBuf<Vec4<S>> relv, drive;
  void ensureFloating() {
    if (dFrame.ptr) return;
    std::vector<FrameDev> h(B);
    for (uint32_t b = 0; b < B; ++b) {
      std::memset(&h[b], 0, sizeof(FrameDev));
      for (int k = 0; k < 3; ++k) h[b].rest_centre[k] = hb[b].restCentre[k];
      h[b].mass = hb[b].mass;
    }
    dFrame.alloc(B);
    dFrame.upload(h.data(), B, st);
    fpart.alloc(size_t(nodeTiles) * FRAME_PART);
    fpart.zero(st);
    relv.alloc(Vp);
    relv.zero(st);
    drive.alloc(Vp);
    drive.zero(st);
    TL_CUDA(cudaStreamSynchronize(st));
  }
  // The frame before the predictor (floatingFrame, solver.cc:3658-3660).
  void frameBegin(uint32_t pass) {
    kFrameMoments<S><<<nodeTiles, TILE, 0, st>>>(view(), pass, 0u);
    check();
    kFrameSolve<S><<<B, TILE, 0, st>>>(view(), pass, 0u);
    check();
    kFrameMoments<S><<<nodeTiles, TILE, 0, st>>>(view(), pass, 1u);
    check();
    kFrameSolve<S><<<B, TILE, 0, st>>>(view(), pass, 1u);
    check();
  }
  // Back to the world after the solve (solver.cc:4265-4340), before kUpdate.
  void frameEnd(uint32_t pass) {
    kFrameMoments<S><<<nodeTiles, TILE, 0, st>>>(view(), pass, 2u);
    check();
    kFrameSolve<S><<<B, TILE, 0, st>>>(view(), pass, 2u);
    check();
    kFrameEnd<S><<<nodeTiles, TILE, 0, st>>>(view(), pass);
    check();
    kFrameSolve<S><<<B, TILE, 0, st>>>(view(), pass, 3u);
    check();
  }
  void frameTurn(uint32_t pass) {
    kFrameTurn<S><<<elemTiles, TILE, 0, st>>>(view(), pass);
    check();
  }
  // TL_FLAG_PROFILE: event pairs around kernel classes, resolved at step end
  bool profiling = false;
  bool tracing = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> evPool;
  std::vector<std::pair<int, size_t>> evUsed;  // (class, pool index)
  cudaEvent_t mark(int cls, bool begin) {
    if (begin) {
      if (evUsed.size() == evPool.size()) {
        cudaEvent_t a, b;
        TL_CUDA(cudaEventCreate(&a));
        TL_CUDA(cudaEventCreate(&b));
        evPool.emplace_back(a, b);
      }
      evUsed.emplace_back(cls, evUsed.size());
      record(evPool[evUsed.back().second].first);
      return evPool[evUsed.back().second].first;
    }
    record(evPool[evUsed.back().second].second);
    return evPool[evUsed.back().second].second;
  }
  // Under stream capture a plain record only orders streams; the external
  // flag makes it an event-record node that fires on every replay.
  bool capturing = false;
  void record(cudaEvent_t e) {
    if (capturing)
      TL_CUDA(cudaEventRecordWithFlags(e, st, cudaEventRecordExternal));
    else
      TL_CUDA(cudaEventRecord(e, st));
  }
  ~System() override {
    if (graphExec) cudaGraphExecDestroy(graphExec);
    for (cudaEvent_t e : xferEvents) cudaEventDestroy(e);
    for (auto& e : evPool) {
      cudaEventDestroy(e.first);
      cudaEventDestroy(e.second);
    }
  }
  PinnedBuf<BodyAccDev> hAcc;
  PinnedBuf<uint32_t> hCount;
  PinnedBuf<CgReportDev> hRep;
  PinnedBuf<GridSyncDev> hSync;
  PinnedBuf<BodyStepDev> hStep;
  PinnedBuf<Vec4<S>> hNode, hNodeV, hNodeA;
  DevBuf<double> dRest;                // [3 Vp] rest positions in FP64, for node arrays converted on the device
  DevBuf<unsigned char> dNodeXfer[3];  // a node array in the caller's layout (position, velocity, acceleration)

  Sys<S> view() {
    Sys<S> s;
    s.bodies = B;
    s.Vp = Vp;
    s.Tp = Tp;
    s.node_tiles = nodeTiles;
    s.elem_tiles = elemTiles;
    s.body = dBody.ptr;
    s.step = dStep.ptr;
    s.mat = dMat.ptr;
    s.flim = dFlim.ptr;
    s.node_tile_body = dNodeTileBody.ptr;
    s.elem_tile_body = dElemTileBody.ptr;
    s.rest4 = rest4.ptr;
    s.anch = anch.ptr;
    s.pres = pres.ptr;
    s.u = u.ptr;
    s.v = v.ptr;
    s.a = a.ptr;
    s.carried = carried.ptr;
    s.shifted = shifted.ptr;
    s.weighted = weighted.ptr;
    s.total = total.ptr;
    s.incr = incr.ptr;
    s.right = right.ptr;
    s.pre0 = pre0.ptr;
    s.pre1 = pre1.ptr;
    s.r = r.ptr;
    s.z = z.ptr;
    s.p = p.ptr;
    s.ap = ap.ptr;
    s.w = w.ptr;
    s.start = start.ptr;
    s.entry = entry.ptr;
    s.tet = tet.ptr;
    s.dm = dm.ptr;
    s.vold = vold.ptr;
    if constexpr (std::is_same_v<S, double>) {  // FP64: the S-typed copies are the FP64 arrays
      s.dms = dm.ptr;
      s.vols = vold.ptr;
    } else {
      s.dms = dms.ptr;
      s.vols = vols.ptr;
    }
    s.lane = lane.ptr;
    s.eyoung = hasEyoung ? eyoung.ptr : nullptr;
    s.op = op.ptr;
    s.orec = orec.ptr;
    s.sell_val = sellReady ? sellVal.ptr : nullptr;
    s.sell_diag = sellReady ? sellDiag.ptr : nullptr;
    s.onorm = onorm.ptr;
    s.tile_meta = tileMeta.ptr;
    s.tile_off = tileOff.ptr;
    s.tile_ent = tileEnt.ptr;
    s.slot_part = slotPart.ptr;
    s.ns_inline = nsInline.ptr;
    s.tile_node = tileNode.ptr;
    s.eloc = eloc.ptr;
    s.ns_start = nsStart.ptr;
    s.ns_slot = nsSlot.ptr;
    s.blk_part = blkPart.ptr;
    s.plast = plast.ptr;
    s.fe = fe.ptr;
    s.de = de.ptr;
    s.de2 = de2.ptr;
    s.ye = ye.ptr;
    s.part = part.ptr;
    s.npart = npart.ptr;
    s.epart = epart.ptr;
    s.loading = loading.ptr;
    s.yielding = yielding.ptr;
    s.acc = acc.ptr;
    s.cg = cg.ptr;
    s.cgrep = cgrep.ptr;
    s.counter = counter.ptr;
    s.sync = sync.ptr;
    s.yflag = yflagPtr;
    s.dtau = hasDamping ? dtau.ptr : nullptr;
    s.dfit = hasDamping ? dfit.ptr : nullptr;
    s.hk = hencky ? hk.ptr : nullptr;
    s.frame = dFrame.ptr;
    s.fpart = fpart.ptr;
    s.relv = relv.ptr;
    s.drive = drive.ptr;
    s.gate = gateBit ? gate.ptr : nullptr;
    s.gate_bit = gateBit;
    return s;
  }

  System(tl_ctx* c, const tl_mesh_desc* descs, uint32_t count) : ctx(c), st(c->stream) {
    B = count;
    bodies = count;
    hb.resize(B);
    bodyHost.resize(B);
    // ---- layout
    uint64_t vp = 0, tp = 0, lanes = 0;
    for (uint32_t b = 0; b < B; ++b) {
      const tl_mesh_desc& d = descs[b];
      if (const char* problem = meshDescProblem(d)) throw StatusError{TL_ERR_ARG, problem};
      BodyDev& bd = bodyHost[b];
      bd.node_begin = uint32_t(vp);
      bd.node_end = uint32_t(vp + d.nodes);
      bd.node_tile_begin = uint32_t(vp / TILE);
      vp += uint64_t(tilesOf(d.nodes)) * TILE;
      bd.node_tile_end = uint32_t(vp / TILE);
      bd.elem_begin = uint32_t(tp);
      bd.elem_end = uint32_t(tp + d.tets);
      bd.elem_tile_begin = uint32_t(tp / TILE);
      tp += uint64_t(tilesOf(d.tets)) * TILE;
      bd.elem_tile_end = uint32_t(tp / TILE);
      lanes += d.lanes + 1;  // + the default lane (material.cc:9-16)
      nodes += d.nodes;
      tets += d.tets;
      if (d.element_youngs) hasEyoung = true;
    }
    if (vp > 0xffffff00ull || tp * 4 > 0xffffff00ull) throw StatusError{TL_ERR_ARG, "system too large"};
    Vp = uint32_t(vp);
    Tp = uint32_t(tp);
    nodeTiles = Vp / TILE;
    elemTiles = Tp / TILE;
    // ---- host staging
    std::vector<Vec4<S>> hRest(Vp, Vec4<S>{0, 0, 0, 0}), hPres(Vp, Vec4<S>{0, 0, 0, 0});
    std::vector<uint8_t> hAnch(Vp, 1u);
    std::vector<uint32_t> hStart(size_t(Vp) + 1, 0u), hEntry(size_t(4) * tets);
    std::vector<uint4> hTet(Tp);
    std::vector<double> hDm(size_t(9) * Tp, 0.0), hVol(Tp, 0.0), hE(hasEyoung ? Tp : 0, 0.0);
    std::vector<S> hDms(size_t(9) * Tp, S(0)), hVols(Tp, S(0));
    std::vector<uint32_t> hLane(Tp, 0u), hNodeTileBody(nodeTiles), hElemTileBody(elemTiles);
    std::vector<MatDev> hMat;
    std::vector<double> laneTau;        // damping weight per material lane
    std::vector<S> hTau(Tp, S(0));      // and per element
    hMat.reserve(lanes);
    for (uint32_t b = 0; b < B; ++b) {
      const tl_mesh_desc& d = descs[b];
      const BodyDev& bd = bodyHost[b];
      HostBody& h = hb[b];
      h.nodes = d.nodes;
      h.tets = d.tets;
      h.rest.assign(d.rest_positions, d.rest_positions + size_t(3) * d.nodes);
      for (uint32_t t = bd.node_tile_begin; t < bd.node_tile_end; ++t) hNodeTileBody[t] = b;
      for (uint32_t t = bd.elem_tile_begin; t < bd.elem_tile_end; ++t) hElemTileBody[t] = b;
      const uint32_t laneBase = uint32_t(hMat.size());
      h.laneBase = laneBase;
      h.lanes = d.lanes;
      for (uint32_t l = 0; l <= d.lanes; ++l) {
        tl_material m = l < d.lanes ? d.materials[l]
                                    : tl_material{1000.0, 0.0, 0.3, 0.0, std::numeric_limits<double>::infinity(), 0.0};
        // stiffnessDamping (factor.cc:755-759): finite and positive, else none
        laneTau.push_back(std::isfinite(m.stiffness_damping) && m.stiffness_damping > 0.0 ? m.stiffness_damping : 0.0);
        const double nu = std::clamp(m.poissons_ratio, 0.0, 0.49);  // material.cc:71-78
        MatDev md;
        md.lam_unit = nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
        md.mu_unit = 1.0 / (2.0 * (1.0 + nu));
        md.youngs = m.youngs_modulus;
        md.yield = m.yield_stress;
        md.hardening = m.hardening_modulus;
        md.yields = (std::isfinite(m.yield_stress) && m.yield_stress > 0.0) ? 1u : 0u;  // material.cc:747-749
        md.pad = 0;
        hMat.push_back(md);
      }
      double centre[3] = {0.0, 0.0, 0.0};
      for (uint32_t n = 0; n < d.nodes; ++n) {
        const uint32_t g = bd.node_begin + n;
        hRest[g] = Vec4<S>{S(d.rest_positions[3 * n]), S(d.rest_positions[3 * n + 1]), S(d.rest_positions[3 * n + 2]),
                           S(d.node_mass[n])};
        // rest centre of the stored (S) rest positions and masses, FP64
        const double m = double(hRest[g].w);
        h.mass += m;
        centre[0] += m * double(hRest[g].x);
        centre[1] += m * double(hRest[g].y);
        centre[2] += m * double(hRest[g].z);
        hAnch[g] = d.anchored[n] ? 1u : 0u;
        h.anyAnchored = h.anyAnchored || d.anchored[n] != 0;
        if (d.prescribed_velocity && d.anchored[n])
          hPres[g] = Vec4<S>{S(d.prescribed_velocity[3 * n]), S(d.prescribed_velocity[3 * n + 1]),
                             S(d.prescribed_velocity[3 * n + 2]), S(0)};
      }
      for (int k = 0; k < 3; ++k) h.restCentre[k] = h.mass > 0.0 ? centre[k] / h.mass : 0.0;
      for (uint32_t t = 0; t < d.tets; ++t) {
        const uint32_t e = bd.elem_begin + t;
        uint32_t q[4];
        for (int k = 0; k < 4; ++k) {
          q[k] = d.tet_nodes[4 * size_t(t) + k] + bd.node_begin;  // in range: meshDescProblem
        }
        hTet[e] = make_uint4(q[0], q[1], q[2], q[3]);
        for (int k = 0; k < 9; ++k) {
          hDm[size_t(k) * Tp + e] = d.rest_inverse[9 * size_t(t) + k];
          hDms[size_t(k) * Tp + e] = S(d.rest_inverse[9 * size_t(t) + k]);
        }
        hVol[e] = d.volume[t];
        hVols[e] = S(d.volume[t]);
        const uint32_t l = d.material[t] < d.lanes ? d.material[t] : d.lanes;
        hLane[e] = laneBase + l;
        hTau[e] = S(laneTau[laneBase + l]);
        if (hTau[e] != S(0)) hasDamping = true;
        if (hMat[laneBase + l].yields) h.anyYields = true;
        if (hasEyoung) hE[e] = d.element_youngs ? d.element_youngs[t] : hMat[laneBase + l].youngs;
        if (b == 0) {  // the first body's mesh, for a solver state's factor
          for (int k = 0; k < 4; ++k) fTets.push_back(d.tet_nodes[4 * size_t(t) + k]);
          fYoungs.push_back(d.element_youngs ? d.element_youngs[t] : (l < d.lanes ? d.materials[l].youngs_modulus : 0.0));
          fPoisson.push_back(l < d.lanes ? d.materials[l].poissons_ratio : 0.3);
          fTau.push_back(laneTau[laneBase + l]);
          fVol.push_back(d.volume[t]);
          for (int k = 0; k < 9; ++k) fDm.push_back(d.rest_inverse[9 * size_t(t) + k]);
        }
      }
      if (b == 0) {
        fAnch.assign(d.anchored, d.anchored + d.nodes);
        fMass.assign(d.node_mass, d.node_mass + d.nodes);
      }
      for (uint32_t t = d.tets; t < bd.elem_tile_end * TILE - bd.elem_begin; ++t) {
        const uint32_t e = bd.elem_begin + t;
        hTet[e] = make_uint4(bd.node_begin, bd.node_begin, bd.node_begin, bd.node_begin);
        hLane[e] = laneBase + d.lanes;
      }
    }
    // ---- CSR node -> (element, corner), ascending element (solver.cc:1065-1101)
    for (uint32_t e = 0; e < Tp; ++e) {
      const uint32_t b = hElemTileBody[e / TILE];
      if (e >= bodyHost[b].elem_end) continue;
      const uint32_t q[4] = {hTet[e].x, hTet[e].y, hTet[e].z, hTet[e].w};
      for (int k = 0; k < 4; ++k) ++hStart[q[k] + 1];
    }
    for (uint32_t n = 0; n < Vp; ++n) hStart[n + 1] += hStart[n];
    {
      std::vector<uint32_t> cursor(hStart.begin(), hStart.end() - 1);
      for (uint32_t e = 0; e < Tp; ++e) {
        const uint32_t b = hElemTileBody[e / TILE];
        if (e >= bodyHost[b].elem_end) continue;
        const uint32_t q[4] = {hTet[e].x, hTet[e].y, hTet[e].z, hTet[e].w};
        for (int k = 0; k < 4; ++k) hEntry[cursor[q[k]]++] = 4 * e + uint32_t(k);
      }
    }
    // ---- device
    dBody.alloc(B);
    dBody.upload(bodyHost.data(), B, st);
    dStep.alloc(B);
    dMat.alloc(hMat.size());
    dMat.upload(hMat.data(), hMat.size(), st);
    // PhysicalMaterial defaults (material.h:16-29): no crush, crush limit 1, no plastic cap
    hFlim.resize(size_t(3) * hMat.size());
    for (size_t l = 0; l < hMat.size(); ++l) {
      hFlim[3 * l] = std::numeric_limits<double>::infinity();
      hFlim[3 * l + 1] = 1.0;
      hFlim[3 * l + 2] = std::numeric_limits<double>::infinity();
    }
    dFlim.alloc(hFlim.size());
    dFlim.upload(hFlim.data(), hFlim.size(), st);
    dNodeTileBody.alloc(nodeTiles);
    dNodeTileBody.upload(hNodeTileBody.data(), nodeTiles, st);
    dElemTileBody.alloc(elemTiles);
    dElemTileBody.upload(hElemTileBody.data(), elemTiles, st);
    rest4.alloc(Vp);
    rest4.upload(hRest.data(), Vp, st);
    pres.alloc(Vp);
    pres.upload(hPres.data(), Vp, st);
    anch.alloc(Vp);
    anch.upload(hAnch.data(), Vp, st);
    for (DevBuf<Vec4<S>>* buf : {&u, &v, &a, &carried, &shifted, &weighted, &total, &incr, &lowest, &right, &pre0,
                                 &pre1, &r, &z, &p, &ap, &w}) {
      buf->alloc(Vp);
      buf->zero(st);
    }
    start.alloc(hStart.size());
    start.upload(hStart.data(), hStart.size(), st);
    entry.alloc(hEntry.size());
    entry.upload(hEntry.data(), hEntry.size(), st);
    tet.alloc(Tp);
    tet.upload(hTet.data(), Tp, st);
    dm.alloc(hDm.size());
    dm.upload(hDm.data(), hDm.size(), st);
    if (sizeof(S) != sizeof(double)) {
      dms.alloc(hDms.size());
      dms.upload(hDms.data(), hDms.size(), st);
      vols.alloc(Tp);
      vols.upload(hVols.data(), Tp, st);
    }
    vold.alloc(Tp);
    vold.upload(hVol.data(), Tp, st);
    lane.alloc(Tp);
    lane.upload(hLane.data(), Tp, st);
    if (hasDamping) {
      dtau.alloc(Tp);
      dtau.upload(hTau.data(), Tp, st);
      dfit.alloc(size_t(20) * Tp);
      dfit.zero(st);
    }
    if (hasEyoung) {
      eyoung.alloc(Tp);
      eyoung.upload(hE.data(), Tp, st);
    }
    op.alloc(size_t(9) * Tp);
    {
      std::vector<S> ident(size_t(9) * Tp, S(0));
      for (int k : {0, 4, 8}) std::fill(ident.begin() + size_t(k) * Tp, ident.begin() + size_t(k + 1) * Tp, S(1));
      op.upload(ident.data(), ident.size(), st);
      TL_CUDA(cudaStreamSynchronize(st));
    }
    orec.alloc(Tp);
    orec.zero(st);
    onorm.alloc(size_t(2) * Tp);
    onorm.zero(st);
    plast.alloc(size_t(2) * Tp);
    plast.zero(st);
    fe.alloc(size_t(4) * Tp);
    de.alloc(size_t(4) * Tp);
    de2.alloc(size_t(4) * Tp);
    ye.alloc(size_t(4) * Tp);
    part.alloc(size_t(4) * nodeTiles);
    npart.alloc(size_t(2) * nodeTiles);
    epart.alloc(elemTiles);
    loading.alloc(B);
    yielding.alloc(B);
    counter.alloc(B);
    counter.zero(st);
    acc.alloc(B);
    cg.alloc(B);
    cg.zero(st);
    cgrep.alloc(B);
    sync.alloc(1);
    sync.zero(st);
    subrec.alloc(size_t(B) * SUBSTEP_RECORDS);
    subrec.zero(st);
    {
      std::vector<double> rest(size_t(3) * Vp, 0.0);
      for (uint32_t b = 0; b < B; ++b)
        std::copy(hb[b].rest.begin(), hb[b].rest.end(), rest.begin() + size_t(3) * bodyHost[b].node_begin);
      dRest.alloc(rest.size());
      dRest.upload(rest.data(), rest.size(), st);
    }
    buildTiles(hTet, hElemTileBody);
    buildSell(hTet, hStart, hEntry, hAnch, hNodeTileBody);
    TL_CUDA(cudaStreamSynchronize(st));
  }

  // Sliced-ELL block structure of the operator (tl_sell.cuh), built on the
  // host by buildSellHost (tl_sell_build.h).
  void buildSell(const std::vector<uint4>& hTet, const std::vector<uint32_t>& hStart,
                 const std::vector<uint32_t>& hEntry, const std::vector<uint8_t>& hAnch,
                 const std::vector<uint32_t>& hNodeTileBody) {
    // one body: its nodes; a batch: every node slot (tile padding rows have
    // no elements and stay zero)
    const uint32_t rows = B == 1 ? bodyHost[0].node_end : Vp;
    if (Tp >= (1u << 28)) return;  // contributor codes hold the element in 28 bits
    static_assert(sizeof(uint4) == 4 * sizeof(uint32_t), "tets are four node ids");
    SellHost h = buildSellHost(rows, reinterpret_cast<const uint32_t*>(hTet.data()), hStart, hEntry);
    const uint32_t slices = h.slices, positions = h.positions, widest = h.widest;
    std::vector<uint32_t>& sliceStart = h.sliceStart;
    std::vector<uint32_t>& groupSlice = h.groupSlice;
    std::vector<uint32_t>& col = h.col;
    std::vector<uint32_t>& cstart = h.cstart;
    std::vector<uint32_t>& centry = h.centry;
    std::vector<uint32_t>& upper = h.upper;
    std::vector<uint32_t>& mirror = h.mirror;
    sellUpperCount = uint32_t(upper.size());
    sellColCache = std::min(widest, SELL_COL_CACHE_MAX);
    // one record per block above the diagonal, in the order of `upper`: its position, its
    // mirror's, its first contributor and (count | row free << 8 | column free << 9 | body << 10)
    std::vector<uint4> urec(std::max<size_t>(upper.size(), 1), make_uint4(0u, 0u, 0u, 0u));
    for (size_t i = 0; i < upper.size(); ++i) {
      const uint32_t pos = upper[i];
      const uint32_t row = groupSlice[pos >> 5] * SELL_ROWS + (pos & 31u), c = col[pos];
      const uint32_t count = cstart[pos + 1] - cstart[pos], body = hNodeTileBody[row / TILE];
      if (count > 0xffu || body >= (1u << 22)) return;  // no assembled operator for such meshes
      urec[i] = make_uint4(pos, mirror[i], cstart[pos],
                           count | (hAnch[row] ? 0u : 1u << 8) | (hAnch[c] ? 0u : 1u << 9) | (body << 10));
    }
    sellUrec.alloc(urec.size());
    sellUrec.upload(urec.data(), urec.size(), st);
    sellDiag.alloc(std::max<size_t>(h.diag.size(), 1));
    sellDiag.upload(h.diag.data(), h.diag.size(), st);
    sellRows = rows;
    sellSlices = slices;
    sellPositions = positions;
    sellStride = std::max(Vp, slices * SELL_ROWS);
    sellSliceStart.alloc(sliceStart.size());
    sellSliceStart.upload(sliceStart.data(), sliceStart.size(), st);
    sellGroupSlice.alloc(groupSlice.size());
    sellGroupSlice.upload(groupSlice.data(), groupSlice.size(), st);
    sellCol.alloc(col.size());
    sellCol.upload(col.data(), col.size(), st);
    sellCentry.alloc(std::max<size_t>(centry.size(), 1));
    sellCentry.upload(centry.data(), centry.size(), st);
    sellVal.alloc(size_t(positions) * 9);
    sellVal.zero(st);  // padding blocks stay zero; kSellAssemble writes the others
    sellVec.alloc(size_t(2) * sellStride);
    sellVec.zero(st);
    for (const void* fn : {(const void*)kPcgSell<S, 2>, (const void*)kPcgSell<S, 4>})
      TL_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sellColBytes())));
    sellPerSmOf[0] = occupancyOf((const void*)kPcgSell<S, 2>, sellColBytes());
    sellPerSmOf[1] = occupancyOf((const void*)kPcgSell<S, 4>, sellColBytes());
    sellPerSm = sellPerSmOf[sellU() == 4u ? 1 : 0];
    // kPcgSell writes four partials per block into one of two halves
    {
      const size_t most = size_t(8) * std::max(sellPerSmOf[0], sellPerSmOf[1]) * ctx->sms;
      if (most > blkPart.count) blkPart.alloc(most);
    }
    // kPcgBatchSell: every batch, and single bodies whose rows exceed one per thread of kPcgSell's grid
    sellP2.alloc(Vp);
    sellP2.zero(st);
    batchSellPerSm = occupancyOf(batchKernel(true), 0);
    if (batchSellPerSm > 0) {
      batchPipePerSm = occupancyOf(batchKernel(false), 0);
      if (batchPipePerSm < 1) throw StatusError{TL_ERR_CUDA, "the pipelined batched PCG cannot be resident"};
    }
    TL_CUDA(cudaStreamSynchronize(st));
    sellReady = sellPerSm > 0 || batchSellPerSm > 0;
  }
  size_t sellColBytes() const { return size_t(sellColCache) * TILE * sizeof(uint32_t); }
  void assembleSell(const Sys<S>& s, const SellDev<S>& g, unsigned blocks, int idx, bool damp, bool tangent,
                    uint32_t pass) {
    if (idx) {
      if (tangent) kSellAssemble<S, 1, true, false><<<blocks, TILE, 0, st>>>(s, g, pass);
      else kSellAssemble<S, 1, false, false><<<blocks, TILE, 0, st>>>(s, g, pass);
    } else if (damp) {
      if (tangent) kSellAssemble<S, 0, true, true><<<blocks, TILE, 0, st>>>(s, g, pass);
      else kSellAssemble<S, 0, false, true><<<blocks, TILE, 0, st>>>(s, g, pass);
    } else {
      if (tangent) kSellAssemble<S, 0, true, false><<<blocks, TILE, 0, st>>>(s, g, pass);
      else kSellAssemble<S, 0, false, false><<<blocks, TILE, 0, st>>>(s, g, pass);
    }
  }
  SellDev<S> sellView() {
    SellDev<S> g;
    g.upper_count = sellUpperCount;
    g.col_cache = sellColCache;
    g.urec = sellUrec.ptr;
    g.rows = sellRows;
    g.slices = sellSlices;
    g.positions = sellPositions;
    g.stride = sellStride;
    g.slice_start = sellSliceStart.ptr;
    g.group_slice = sellGroupSlice.ptr;
    g.col = sellCol.ptr;
    g.centry = sellCentry.ptr;
    g.val = sellVal.ptr;
    g.vec = sellVec.ptr;
    return g;
  }
  // Grid of kPcgSell: the occupancy (capped by tl_system_tune while every
  // block still has at most one slice per warp), or 0 when the rows do not
  // fit one per thread.
  // Whether this system's PCG runs on the assembled matrix.  TL_SOLVER_AUTO
  // assembles batches, and single bodies large enough for the per-solve
  // assembly to pay (measured on a B200: element-by-element 17% faster at
  // 3,072 tets, even at 24,576, assembled 1.6x faster at 393,216).
  bool assembledForm() const {
    if (!sellReady || solverForm == TL_SOLVER_ELEMENTWISE) return false;
    return B > 1 || solverForm == TL_SOLVER_ASSEMBLED || solverForm == TL_SOLVER_ASSEMBLED_TWO_PHASE ||
           solverForm == TL_SOLVER_ASSEMBLED_PIPELINED || bodyHost[0].elem_end >= SELL_AUTO_MIN_TETS;
  }
  int sellGrid() const {
    if (B != 1 || sellPerSm < 1 || !assembledForm()) return 0;
    const int full = std::min<int>(sellPerSm * ctx->sms, int(sellSlices));
    const int capped = tuneBlocksPerSm ? std::min<int>(std::min<int>(sellPerSm, int(tuneBlocksPerSm)) * ctx->sms,
                                                       int(sellSlices))
                                       : full;
    const auto fits = [&](int g) { return g > 0 && uint64_t(sellSlices) <= uint64_t(g) * SELL_SLICES_PER_BLOCK; };
    if (fits(capped)) return capped;
    return fits(full) ? full : 0;
  }

  // Two-level assembly structures: per element tile the distinct nodes it
  // touches (its slots, ascending node) with a tile-local CSR of the
  // (local element, corner) codes in ascending element order; per node the
  // slots holding its partial sums, in ascending tile order.
  void buildTiles(const std::vector<uint4>& hTet, const std::vector<uint32_t>& hElemTileBody) {
    std::vector<uint2> meta(elemTiles);
    std::vector<uint16_t> off(size_t(elemTiles) * TILE_OFF_STRIDE, 0), ent(size_t(elemTiles) * 4 * TILE, 0);
    std::vector<uint32_t> slotNode;
    std::vector<uint16_t> cornerSlot(size_t(4) * Tp, 0);
    std::vector<std::pair<uint32_t, uint32_t>> items;  // (node, code)
    for (uint32_t t = 0; t < elemTiles; ++t) {
      const BodyDev& bd = bodyHost[hElemTileBody[t]];
      const uint32_t e0 = t * TILE, e1 = std::min<uint32_t>(e0 + TILE, bd.elem_end);
      items.clear();
      for (uint32_t e = e0; e < e1; ++e) {
        const uint32_t q[4] = {hTet[e].x, hTet[e].y, hTet[e].z, hTet[e].w};
        for (uint32_t c = 0; c < 4; ++c) items.emplace_back(q[c], 4 * (e - e0) + c);
      }
      std::sort(items.begin(), items.end());
      const uint32_t base = uint32_t(slotNode.size());
      uint16_t* o = off.data() + size_t(t) * TILE_OFF_STRIDE;
      uint16_t* en = ent.data() + size_t(t) * 4 * TILE;
      uint32_t local = 0;
      for (size_t k = 0; k < items.size(); ++k) {
        if (k == 0 || items[k].first != items[k - 1].first) {
          o[local++] = uint16_t(k);
          slotNode.push_back(items[k].first);
        }
        en[k] = uint16_t(items[k].second);
        // corner (element, c) of this item reads local node (local - 1)
        const uint32_t le = items[k].second >> 2, c = items[k].second & 3u;
        cornerSlot[size_t(e0 + le) * 4 + c] = uint16_t(local - 1);
      }
      o[local] = uint16_t(items.size());
      meta[t] = make_uint2(base, local);
    }
    const size_t slots = slotNode.size();
    std::vector<uint32_t> start(size_t(Vp) + 1, 0), list(slots);
    for (uint32_t n : slotNode) ++start[n + 1];
    for (uint32_t n = 0; n < Vp; ++n) start[n + 1] += start[n];
    {
      std::vector<uint32_t> cursor(start.begin(), start.end() - 1);
      for (size_t k = 0; k < slots; ++k) list[cursor[slotNode[k]]++] = uint32_t(k);  // slots ascend with tiles
    }
    // the first 8 slots of each node inline, the rest in an overflow CSR
    std::vector<uint4> inl(size_t(2) * Vp, make_uint4(NO_SLOT, NO_SLOT, NO_SLOT, NO_SLOT));
    std::vector<uint32_t> ostart(size_t(Vp) + 1, 0), olist;
    for (uint32_t n = 0; n < Vp; ++n) {
      uint32_t ids[8] = {NO_SLOT, NO_SLOT, NO_SLOT, NO_SLOT, NO_SLOT, NO_SLOT, NO_SLOT, NO_SLOT};
      for (uint32_t k = start[n]; k < start[n + 1]; ++k) {
        if (k - start[n] < 8) ids[k - start[n]] = list[k];
        else olist.push_back(list[k]);
      }
      inl[n] = make_uint4(ids[0], ids[1], ids[2], ids[3]);
      inl[size_t(Vp) + n] = make_uint4(ids[4], ids[5], ids[6], ids[7]);
      ostart[n + 1] = uint32_t(olist.size());
    }
    tileMeta.alloc(elemTiles);
    tileMeta.upload(meta.data(), elemTiles, st);
    tileOff.alloc(off.size());
    tileOff.upload(off.data(), off.size(), st);
    tileEnt.alloc(ent.size());
    tileEnt.upload(ent.data(), ent.size(), st);
    slotPart.alloc(std::max<size_t>(slots, 1));
    tileNode.alloc(std::max<size_t>(slots, 1));
    tileNode.upload(slotNode.data(), slots, st);
    {
      std::vector<uint2> loc(Tp);
      for (uint32_t e = 0; e < Tp; ++e) {
        const uint16_t* q = cornerSlot.data() + size_t(e) * 4;
        loc[e] = make_uint2(uint32_t(q[0]) | (uint32_t(q[1]) << 16), uint32_t(q[2]) | (uint32_t(q[3]) << 16));
      }
      eloc.alloc(Tp);
      eloc.upload(loc.data(), Tp, st);
      TL_CUDA(cudaStreamSynchronize(st));
    }
    nsInline.alloc(inl.size());
    nsInline.upload(inl.data(), inl.size(), st);
    nsStart.alloc(ostart.size());
    nsStart.upload(ostart.data(), ostart.size(), st);
    nsSlot.alloc(std::max<size_t>(olist.size(), 1));
    nsSlot.upload(olist.data(), olist.size(), st);
    TL_CUDA(cudaStreamSynchronize(st));
    // resident blocks per SM of each cooperative kernel variant (the grid is
    // that times the SM count, capped by tl_system_tune and the tile counts)
    // (the batched variants take their operator stage as dynamic shared memory)
    auto perSm = [&](const void* fn, size_t dyn) {
      TL_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn)));
      int n = 0;
      TL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, TILE, dyn));
      if (n < 1) throw StatusError{TL_ERR_CUDA, "PCG kernel cannot be resident"};
      return n;
    };
    // the element pass's shared-memory stage is above the default 48 KB
    for (const void* fn : {(const void*)kElement<S, 0>, (const void*)kElement<S, 1>, (const void*)kElement<S, 0, true>})
      TL_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(elementStageBytes<S>())));
    // the element pass runs as a resident grid that walks the tiles (no block launches between rounds)
    elementGrid[0] = std::min<uint32_t>(std::max<uint32_t>(elemTiles, 1u), uint32_t(perSm((const void*)kElement<S, 0>, elementStageBytes<S>())) * ctx->sms);
    elementGrid[1] = std::min<uint32_t>(std::max<uint32_t>(elemTiles, 1u), uint32_t(perSm((const void*)kElement<S, 1>, elementStageBytes<S>())) * ctx->sms);
    elementGrid[2] =
        std::min<uint32_t>(std::max<uint32_t>(elemTiles, 1u), uint32_t(perSm((const void*)kElement<S, 0, true>, elementStageBytes<S>())) * ctx->sms);
    pcg1PerSm[0][0] = perSm((const void*)kPcg1<S, 0, false>, sizeof(TileCache));
    pcg1PerSm[0][1] = perSm((const void*)kPcg1<S, 0, true>, sizeof(TileCache));
    pcg1PerSm[1][0] = perSm((const void*)kPcg1<S, 1, false>, sizeof(TileCache));
    pcg1PerSm[1][1] = perSm((const void*)kPcg1<S, 1, true>, sizeof(TileCache));
    batchPerSm[0][0] = perSm((const void*)kPcgBatch<S, 0, false>, pipeBytes<S, 0, false>());
    batchPerSm[0][1] = perSm((const void*)kPcgBatch<S, 0, true>, pipeBytes<S, 0, true>());
    batchPerSm[1][0] = perSm((const void*)kPcgBatch<S, 1, false>, pipeBytes<S, 1, false>());
    batchPerSm[1][1] = perSm((const void*)kPcgBatch<S, 1, true>, pipeBytes<S, 1, true>());
    if (hasDamping) {
      pcg1DampPerSm[0] = perSm((const void*)kPcg1<S, 0, false, true>, sizeof(TileCache));
      pcg1DampPerSm[1] = perSm((const void*)kPcg1<S, 0, true, true>, sizeof(TileCache));
      batchDampPerSm[0] = perSm((const void*)kPcgBatch<S, 0, false, true>, pipeBytes<S, 0, false>());
      batchDampPerSm[1] = perSm((const void*)kPcgBatch<S, 0, true, true>, pipeBytes<S, 0, true>());
    }
    int most = 0;
    for (auto& row : pcg1PerSm)
      for (int n : row) most = std::max(most, n * ctx->sms);
    for (int n : pcg1DampPerSm) most = std::max(most, n * ctx->sms);
    blkPart.alloc(size_t(3) * most);
  }

  // ------------------------------------------------------------- state ----

  template <class H>
  void setNodes(const BodyDev& bd, const HostBody& h, DevBuf<Vec4<S>>& dst, const H* src, bool displacement) {
    stageNodes(bd, h, dst, src, displacement, hNode);
    TL_CUDA(cudaStreamSynchronize(st));
  }
  // Converts one node array into its pinned stage and queues the upload (the
  // stage must not be reused before the stream has passed the copy).
  template <class H>
  void stageNodes(const BodyDev& bd, const HostBody& h, DevBuf<Vec4<S>>& dst, const H* src, bool displacement,
                  PinnedBuf<Vec4<S>>& buf) {
    if (pinnedHost(src)) {  // the caller pinned its buffer: one DMA, converted on the device
      if (!h.nodes) return;
      DevBuf<unsigned char>& xfer = nodeXfer(buf);
      const size_t bytes = size_t(3) * h.nodes * sizeof(H);
      if (xfer.count < bytes) xfer.alloc(bytes);
      TL_CUDA(cudaMemcpyAsync(xfer.ptr, src, bytes, cudaMemcpyHostToDevice, st));
      kNodeStateIn<S, H><<<(h.nodes + TILE - 1) / TILE, TILE, 0, st>>>(
          dst.ptr + bd.node_begin, reinterpret_cast<const H*>(xfer.ptr),
          displacement ? dRest.ptr + size_t(3) * bd.node_begin : nullptr, h.nodes);
      check();
      return;
    }
    Vec4<S>* stage = buf.get(h.nodes);
    parallelFor(h.nodes, [&](size_t n0, size_t n1) {
      for (size_t n = n0; n < n1; ++n) {
        double x = double(src[3 * n]), y = double(src[3 * n + 1]), zz = double(src[3 * n + 2]);
        if (displacement) {
          x -= h.rest[3 * n];
          y -= h.rest[3 * n + 1];
          zz -= h.rest[3 * n + 2];
        }
        stage[n] = Vec4<S>{S(x), S(y), S(zz), S(0)};
      }
    });
    dst.upload(stage, h.nodes, st, bd.node_begin);
  }
  // The device scratch that goes with a node array's pinned stage.
  DevBuf<unsigned char>& nodeXfer(const PinnedBuf<Vec4<S>>& buf) {
    return dNodeXfer[&buf == &hNode ? 0 : &buf == &hNodeV ? 1 : 2];
  }
  // Converts a node array on the device and copies it straight into the
  // caller's page-locked buffer.
  template <class H>
  void fetchNodesDirect(const BodyDev& bd, const HostBody& h, const DevBuf<Vec4<S>>& src, H* dst, bool displacement,
                        const PinnedBuf<Vec4<S>>& buf) {
    if (!h.nodes) return;
    DevBuf<unsigned char>& xfer = nodeXfer(buf);
    const size_t bytes = size_t(3) * h.nodes * sizeof(H);
    if (xfer.count < bytes) xfer.alloc(bytes);
    kNodeStateOut<S, H><<<(h.nodes + TILE - 1) / TILE, TILE, 0, st>>>(
        reinterpret_cast<H*>(xfer.ptr), src.ptr + bd.node_begin,
        displacement ? dRest.ptr + size_t(3) * bd.node_begin : nullptr, h.nodes);
    check();
    TL_CUDA(cudaMemcpyAsync(dst, xfer.ptr, bytes, cudaMemcpyDeviceToHost, st));
  }
  template <class H>
  void getNodes(const BodyDev& bd, const HostBody& h, const DevBuf<Vec4<S>>& src, H* dst, bool displacement) {
    Vec4<S>* stage = hNode.get(h.nodes);
    src.download(stage, h.nodes, st, bd.node_begin);
    TL_CUDA(cudaStreamSynchronize(st));
    unstageNodes(h, stage, dst, displacement);
  }
  template <class H>
  void unstageNodes(const HostBody& h, const Vec4<S>* stage, H* dst, bool displacement) {
    parallelFor(h.nodes, [&](size_t n0, size_t n1) {
      for (size_t n = n0; n < n1; ++n) {
        double x = double(stage[n].x), y = double(stage[n].y), zz = double(stage[n].z);
        if (displacement) {
          x += h.rest[3 * n];
          y += h.rest[3 * n + 1];
          zz += h.rest[3 * n + 2];
        }
        dst[3 * n] = H(x);
        dst[3 * n + 1] = H(y);
        dst[3 * n + 2] = H(zz);
      }
    });
  }
  // Element state crosses the host boundary in the caller's layout: a
  // parallel memcpy between the caller's buffer and pinned staging, one copy
  // each way, and the plane layout converted on the device (kElemStateIn /
  // kElemStateOut).  Measured on a B200 box, this beat copies straight from
  // the caller's pageable buffers by 15-25% per tl_step_host.
  PinnedBuf<unsigned char> hXfer;  // element state in the caller's layout, host side
  DevBuf<unsigned char> dXfer;     // and device side
  template <class H> void elemStaging(size_t values, H*& host, H*& dev) {
    const size_t bytes = values * sizeof(H);
    if (dXfer.count < bytes) dXfer.alloc(bytes);
    host = reinterpret_cast<H*>(hXfer.get(bytes));
    dev = reinterpret_cast<H*>(dXfer.ptr);
  }
  // Host <-> staging copies and DMA in chunks of XFER_CHUNK bytes: each
  // chunk's DMA runs while the host copies the next one (uploads), or the
  // host copies a chunk out while the later ones are still in flight
  // (downloads, one event per chunk).
  static constexpr size_t XFER_CHUNK = size_t(4) << 20;
  std::vector<cudaEvent_t> xferEvents;
  void upload(unsigned char* dev, unsigned char* stage, const unsigned char* src, size_t bytes) {
    if (pinnedHost(src)) {  // the caller pinned its buffer (tl_host_register): one DMA, no staging
      TL_CUDA(cudaMemcpyAsync(dev, src, bytes, cudaMemcpyHostToDevice, st));
      return;
    }
    for (size_t o = 0; o < bytes; o += XFER_CHUNK) {
      const size_t n = std::min(XFER_CHUNK, bytes - o);
      parallelCopy(stage + o, src + o, n);
      TL_CUDA(cudaMemcpyAsync(dev + o, stage + o, n, cudaMemcpyHostToDevice, st));
    }
  }
  void queueDownload(unsigned char* stage, const unsigned char* dev, size_t bytes) {
    const size_t chunks = (bytes + XFER_CHUNK - 1) / XFER_CHUNK;
    while (xferEvents.size() < chunks) {
      cudaEvent_t e;
      TL_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      xferEvents.push_back(e);
    }
    for (size_t c = 0; c < chunks; ++c) {
      const size_t o = c * XFER_CHUNK, n = std::min(XFER_CHUNK, bytes - o);
      TL_CUDA(cudaMemcpyAsync(stage + o, dev + o, n, cudaMemcpyDeviceToHost, st));
      TL_CUDA(cudaEventRecord(xferEvents[c], st));
    }
  }
  template <class H>
  void setElems(const BodyDev& bd, const HostBody& h, const H* rot, const H* plastic) {
    const uint32_t T = h.tets;
    const size_t nR = rot ? size_t(9) * T : 0, nP = plastic ? size_t(10) * T : 0;
    if (!nR && !nP) return;
    H *stage, *dev;
    elemStaging<H>(nR + nP, stage, dev);
    auto bytes = [](auto* p) { return reinterpret_cast<unsigned char*>(p); };
    if (rot) upload(bytes(dev), bytes(stage), reinterpret_cast<const unsigned char*>(rot), nR * sizeof(H));
    if (plastic)
      upload(bytes(dev + nR), bytes(stage + nR), reinterpret_cast<const unsigned char*>(plastic), nP * sizeof(H));
    kElemStateIn<S, H><<<(T + TILE - 1) / TILE, TILE, 0, st>>>(view(), bd.elem_begin, T, rot ? dev : nullptr,
                                                               plastic ? dev + nR : nullptr);
    check();
  }
  // Queues the conversion of a body's element state and its download into
  // the pinned staging.
  // With direct set (every requested caller buffer pinned), the state goes
  // straight into the caller's buffers and getElems has nothing to copy.
  template <class H>
  void fetchElems(const BodyDev& bd, const HostBody& h, H* rot, H* plastic, bool direct) {
    const uint32_t T = h.tets;
    const size_t nR = rot ? size_t(9) * T : 0, nP = plastic ? size_t(10) * T : 0;
    if (!nR && !nP) return;
    H *stage, *dev;
    elemStaging<H>(nR + nP, stage, dev);
    kElemStateOut<S, H><<<(T + TILE - 1) / TILE, TILE, 0, st>>>(view(), bd.elem_begin, T, rot ? dev : nullptr,
                                                                plastic ? dev + nR : nullptr);
    check();
    if (direct) {
      if (nR) TL_CUDA(cudaMemcpyAsync(rot, dev, nR * sizeof(H), cudaMemcpyDeviceToHost, st));
      if (nP) TL_CUDA(cudaMemcpyAsync(plastic, dev + nR, nP * sizeof(H), cudaMemcpyDeviceToHost, st));
      return;
    }
    queueDownload(reinterpret_cast<unsigned char*>(stage), reinterpret_cast<const unsigned char*>(dev),
                  (nR + nP) * sizeof(H));
  }
  // Copies the fetched element state out, chunk by chunk as it arrives.
  template <class H>
  void getElems(const HostBody& h, H* rot, H* plastic) {
    const uint32_t T = h.tets;
    const size_t nR = rot ? size_t(9) * T : 0, nP = plastic ? size_t(10) * T : 0;
    const unsigned char* stage = hXfer.ptr;
    if (!nR && !nP) return;
    // the staging holds [rotations][plastic]; chunks may straddle the two
    const size_t total = (nR + nP) * sizeof(H);
    for (size_t o = 0, c = 0; o < total; o += XFER_CHUNK, ++c) {
      TL_CUDA(cudaEventSynchronize(xferEvents[c]));
      const size_t end = std::min(total, o + XFER_CHUNK), split = nR * sizeof(H);
      if (o < split) parallelCopy(reinterpret_cast<unsigned char*>(rot) + o, stage + o, std::min(end, split) - o);
      if (end > split) {
        const size_t from = std::max(o, split);
        parallelCopy(reinterpret_cast<unsigned char*>(plastic) + (from - split), stage + from, end - from);
      }
    }
  }

  void stateSet(uint32_t b, int32_t dtype, const void* x, const void* vv, const void* aa, const void* rot,
                const void* pl) override {
    const BodyDev& bd = bodyHost[b];
    const HostBody& h = hb[b];
    // every array has its own pinned stage: conversions overlap the uploads
    // queued before them, and the stream is waited on once
    if (dtype == TL_DTYPE_F64) {
      if (x) stageNodes(bd, h, u, static_cast<const double*>(x), true, hNode);
      if (vv) stageNodes(bd, h, v, static_cast<const double*>(vv), false, hNodeV);
      if (aa) stageNodes(bd, h, a, static_cast<const double*>(aa), false, hNodeA);
      setElems(bd, h, static_cast<const double*>(rot), static_cast<const double*>(pl));
    } else {
      if (x) stageNodes(bd, h, u, static_cast<const float*>(x), true, hNode);
      if (vv) stageNodes(bd, h, v, static_cast<const float*>(vv), false, hNodeV);
      if (aa) stageNodes(bd, h, a, static_cast<const float*>(aa), false, hNodeA);
      setElems(bd, h, static_cast<const float*>(rot), static_cast<const float*>(pl));
    }
    TL_CUDA(cudaStreamSynchronize(st));
  }
  void stateGet(uint32_t b, int32_t dtype, void* x, void* vv, void* aa, void* rot, void* pl) override {
    const BodyDev& bd = bodyHost[b];
    const HostBody& h = hb[b];
    // queue every download, wait once, then convert; a page-locked caller
    // buffer gets its array converted on the device and copied straight in
    auto direct_node = [&](void* p) { return p && pinnedHost(p); };
    const bool dx = direct_node(x), dv = direct_node(vv), da = direct_node(aa);
    Vec4<S>* sx = x && !dx ? hNode.get(h.nodes) : nullptr;
    Vec4<S>* sv = vv && !dv ? hNodeV.get(h.nodes) : nullptr;
    Vec4<S>* sa = aa && !da ? hNodeA.get(h.nodes) : nullptr;
    if (sx) u.download(sx, h.nodes, st, bd.node_begin);
    if (sv) v.download(sv, h.nodes, st, bd.node_begin);
    if (sa) a.download(sa, h.nodes, st, bd.node_begin);
    if (dtype == TL_DTYPE_F64) {
      if (dx) fetchNodesDirect(bd, h, u, static_cast<double*>(x), true, hNode);
      if (dv) fetchNodesDirect(bd, h, v, static_cast<double*>(vv), false, hNodeV);
      if (da) fetchNodesDirect(bd, h, a, static_cast<double*>(aa), false, hNodeA);
    } else {
      if (dx) fetchNodesDirect(bd, h, u, static_cast<float*>(x), true, hNode);
      if (dv) fetchNodesDirect(bd, h, v, static_cast<float*>(vv), false, hNodeV);
      if (da) fetchNodesDirect(bd, h, a, static_cast<float*>(aa), false, hNodeA);
    }
    const bool direct = (!rot || pinnedHost(rot)) && (!pl || pinnedHost(pl));
    if (dtype == TL_DTYPE_F64)
      fetchElems<double>(bd, h, static_cast<double*>(rot), static_cast<double*>(pl), direct);
    else
      fetchElems<float>(bd, h, static_cast<float*>(rot), static_cast<float*>(pl), direct);
    // element state is copied out chunk by chunk as it arrives; the node
    // records were queued first, so they have arrived once the stream ends
    if (!direct) {
      if (dtype == TL_DTYPE_F64) getElems(h, static_cast<double*>(rot), static_cast<double*>(pl));
      else getElems(h, static_cast<float*>(rot), static_cast<float*>(pl));
    }
    TL_CUDA(cudaStreamSynchronize(st));
    if (dtype == TL_DTYPE_F64) {
      if (sx) unstageNodes(h, sx, static_cast<double*>(x), true);
      if (sv) unstageNodes(h, sv, static_cast<double*>(vv), false);
      if (sa) unstageNodes(h, sa, static_cast<double*>(aa), false);
    } else {
      if (sx) unstageNodes(h, sx, static_cast<float*>(x), true);
      if (sv) unstageNodes(h, sv, static_cast<float*>(vv), false);
      if (sa) unstageNodes(h, sa, static_cast<float*>(aa), false);
    }
  }

  // ---------------------------------------------------------- launches ----

  void check() {
    TL_CUDA(cudaGetLastError());
    ++launches;
  }
  void element(int law, const Vec4<S>* base, const Vec4<S>* dir, uint32_t pass, uint32_t mode, double margin) {
    if (!(mode & EM_COMMIT)) {  // the counters describe the last assemble, not commitPlastic
      loading.zero(st);
      yielding.zero(st);
    }
    if (profiling) mark(0, true);
    if (std::any_of(hb.begin(), hb.end(), [](const HostBody& h) { return h.anyYields; })) mode |= EM_YIELDING;
    const bool damps = hasDamping && law == TL_LAW_COROTATED && !(mode & EM_COMMIT) && !evaluating;
    if (law == TL_LAW_SNH)
      kElement<S, 1><<<elementGrid[1], TILE, elementStageBytes<S>(), st>>>(view(), base, dir, pass, mode, margin);
    else if (hencky)
      kElement<S, 0, true><<<elementGrid[2], TILE, elementStageBytes<S>(), st>>>(view(), base, dir, pass, mode, margin);
    else
      kElement<S, 0><<<elementGrid[0], TILE, elementStageBytes<S>(), st>>>(view(), base, dir, pass, mode, margin);
    check();
    if (damps) {
      kDamping<S><<<elemTiles, TILE, 0, st>>>(view(), base, dir, pass);
      check();
    }
    if (profiling) mark(0, false);
  }
  void nodeAssemble(const Vec4<S>* taken, uint32_t pass) {
    if (profiling) mark(1, true);
    kNodeAssemble<S><<<nodeTiles, TILE, 0, st>>>(view(), taken, pass);
    check();
    if (profiling) mark(1, false);
  }
  // tl_system_expire_wait: the step's PCG solve number expireSolve (from 0)
  // is preceded by the bounded-wait self test on this system's barrier word.
  int64_t expireSolve = -1;
  uint64_t solveCount = 0;  // PCG solves issued in the current step
  void pcg(int law, Vec4<S>* X, uint32_t pass, bool x0zero, bool tangent) {
    if (expireSolve >= 0 && solveCount == uint64_t(expireSolve)) {
      // the previous solve left its arrivals in the counter: start the wait from zero
      TL_CUDA(cudaMemsetAsync(&sync.ptr->arrive, 0, sizeof(unsigned int), st));
      kWaitLimitCheck<<<1, TILE, 0, st>>>(sync.ptr);
      check();
      expireSolve = -1;
    }
    ++solveCount;
    if (factorOn && fPrepared && fHost.ready) {  // a solver state with a factor: kPcgFactor
      pcgFactor(law, X, pass, x0zero, tangent);
      return;
    }
    kPcgPrepare<S><<<1, TILE, 0, st>>>(view(), pass);
    check();
    Sys<S> s = view();
    uint32_t ps = pass, xz = x0zero ? 1u : 0u, tg = tangent ? 1u : 0u;
    const int idx = law == TL_LAW_SNH ? 1 : 0;
    const size_t dyn = idx ? (tangent ? pipeBytes<S, 1, true>() : pipeBytes<S, 1, false>())
                           : (tangent ? pipeBytes<S, 0, true>() : pipeBytes<S, 0, false>());
    const bool damp = hasDamping && idx == 0;
    const int sellG = sellGrid();
    if (sellG > 0) {  // single body: assembled block matrix, pipelined PCG
      SellDev<S> g = sellView();
      const unsigned blocks = (sellUpperCount + TILE - 1) / TILE;
      if (profiling) mark(1, true);  // the operator assembly counts as assembly time
      assembleSell(s, g, blocks, idx, damp, tangent, ps);
      check();
      ++launches;
      if (profiling) {
        mark(1, false);
        mark(2, true);
      }
      void* args[] = {&s, &g, &X, &xz, &tg};
      TL_CUDA(cudaLaunchCooperativeKernel(sellKernel(), dim3(sellG), dim3(TILE), args, sellColBytes(), st));
    } else if (B == 1) {  // single body, element by element: two-level assembly, per-block partials
      if (profiling) mark(2, true);
      void* args[] = {&s, &X, &xz};
      const void* fn = idx ? (tangent ? (const void*)kPcg1<S, 1, true> : (const void*)kPcg1<S, 1, false>)
                           : damp ? (tangent ? (const void*)kPcg1<S, 0, true, true> : (const void*)kPcg1<S, 0, false, true>)
                                  : (tangent ? (const void*)kPcg1<S, 0, true> : (const void*)kPcg1<S, 0, false>);
      const int perSm = damp ? pcg1DampPerSm[tangent ? 1 : 0] : pcg1PerSm[idx][tangent ? 1 : 0];
      TL_CUDA(cudaLaunchCooperativeKernel(fn, dim3(gridOf(perSm)), dim3(TILE), args,
                                          sizeof(TileCache), st));
    } else if (assembledForm() && batchSellPerSm > 0) {  // batch, or a body too large for kPcgSell
      SellDev<S> g = sellView();
      const unsigned blocks = (sellUpperCount + TILE - 1) / TILE;
      if (profiling) mark(1, true);
      assembleSell(s, g, blocks, idx, damp, tangent, ps);
      check();
      ++launches;
      if (profiling) {
        mark(1, false);
        mark(2, true);
      }
      Vec4<S>* p2 = sellP2.ptr;
      // the batch's order: measured on 512 uneven bodies solved to 1e-6, the pipelined
      // order (FP64 recurrences) is the faster in FP64 and the two-phase one in FP32-mixed
      const bool twoPhase = solverForm == TL_SOLVER_ASSEMBLED_TWO_PHASE ||
                            (solverForm != TL_SOLVER_ASSEMBLED_PIPELINED && sizeof(S) == 4);
      int perSm = twoPhase ? batchSellPerSm : batchPipePerSm;
      int grid = std::max(1, std::min(perSm * ctx->sms, int(nodeTiles)));
      // the block's slot table: body and row count of each of its tiles
      size_t slotBytes = size_t(2) * sizeof(uint32_t) * ((nodeTiles + grid - 1) / grid);
      if (slotBytes > 48 * 1024) throw StatusError{TL_ERR_UNSUPPORTED, "too many node tiles for the batched PCG grid"};
      if (slotBytes > 1024) {  // a large table may cost residency: size the cooperative grid with it
        const int withTable = occupancyOf(batchKernel(twoPhase), slotBytes);
        if (withTable < 1) throw StatusError{TL_ERR_UNSUPPORTED, "the batched PCG grid cannot be resident"};
        if (withTable < perSm) {
          perSm = withTable;
          grid = std::max(1, std::min(perSm * ctx->sms, int(nodeTiles)));
          slotBytes = size_t(2) * sizeof(uint32_t) * ((nodeTiles + grid - 1) / grid);
          if (occupancyOf(batchKernel(twoPhase), slotBytes) < perSm)
            throw StatusError{TL_ERR_UNSUPPORTED, "the batched PCG grid cannot be resident"};
        }
      }
      if (twoPhase) {
        void* args[] = {&s, &g, &X, &p2, &ps, &xz, &tg};
        TL_CUDA(cudaLaunchCooperativeKernel(batchKernel(true), dim3(grid), dim3(TILE), args, slotBytes, st));
      } else {
        if (!pipeState.ptr) pipeState.alloc(size_t(8) * Vp);
        Vec4<double>* state = pipeState.ptr;
        void* args[] = {&s, &g, &X, &state, &ps, &xz, &tg};
        TL_CUDA(cudaLaunchCooperativeKernel(batchKernel(false), dim3(grid), dim3(TILE), args, slotBytes, st));
      }
    } else {  // batch: two-level assembly, per-body scalars
      if (profiling) mark(2, true);
      void* args[] = {&s, &X, &ps, &xz};
      const void* fn =
          idx ? (tangent ? (const void*)kPcgBatch<S, 1, true> : (const void*)kPcgBatch<S, 1, false>)
              : damp ? (tangent ? (const void*)kPcgBatch<S, 0, true, true> : (const void*)kPcgBatch<S, 0, false, true>)
                     : (tangent ? (const void*)kPcgBatch<S, 0, true> : (const void*)kPcgBatch<S, 0, false>);
      const int perSm = damp ? batchDampPerSm[tangent ? 1 : 0] : batchPerSm[idx][tangent ? 1 : 0];
      TL_CUDA(cudaLaunchCooperativeKernel(fn, dim3(gridOf(perSm)), dim3(TILE), args, dyn, st));
    }
    ++launches;
    if (profiling) mark(2, false);
    if (tracing) {
      uint32_t taken = 0;
      TL_CUDA(cudaMemcpyAsync(&taken, &cg.ptr[0].taken, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
      TL_CUDA(cudaStreamSynchronize(st));
      trace.push_back(taken);
    }
  }
  // ------------------------------------------------------ solver state ----
  // The caller-held solver state (DeformableSolverState, factor.h:205-210)
  // of a one-body system: its factor (made on the host, tl_factor_host.h),
  // the factor in the device layout of kPcgFactor, the FactorReference and
  // the SolverStats.
  bool factorOn = false;
  uint32_t factorBudget = 32u;
  BlockFactor fHost;
  double fStep = 0.0, fInertia = 1.0;  // FactorReference::step, ::inertia
  bool fPrepared = false;              // a factor is prepared for the current substep
  uint32_t fBudget = 0u;               // the iteration budget of the substep's factored solves
  tl_factor_stats fStats{};
  float fMean = 0.0f;                  // SolverStats::meanIterations is a float
  std::vector<uint32_t> fTets;         // body 0: tets, per-tet Young's modulus and Poisson ratio, anchors, masses
  std::vector<double> fYoungs, fPoisson, fMass, fTau, fVol, fDm;  // fDm: Dm^-1 row-major
  std::vector<uint8_t> fAnch;
  DevBuf<uint32_t> dfPerm, dfIperm, dfRowStart, dfRowCol, dfColStart, dfColRow, dfFlags, dfTicket, dfSnStart,
      dfRowSplit, dfColSplit;
  DevBuf<int32_t> dfSnChild, dfSnParent;
  DevBuf<double> dfRowBlk, dfColBlk, dfDiagInv, dfFrame, dfPart;
  DevBuf<Vec4<double>> dfY, dfW, dfRef, dfRhs;
  DevBuf<Vec4<S>> dfR, dfD, dfQ, dfZ, dfRestart;
  int factorPerSm = 0;

  void useFactor(uint32_t enable, uint32_t budget) override {
    if (!enable) {
      factorOn = false;
      return;
    }
    if (B != 1) throw StatusError{TL_ERR_UNSUPPORTED, "a solver state is held for one-body systems"};
    if (!sellReady) throw StatusError{TL_ERR_UNSUPPORTED, "the factored PCG needs the assembled operator"};
    if (hencky) throw StatusError{TL_ERR_UNSUPPORTED, "the factor is made for the small-strain path"};
    factorOn = true;
    factorBudget = budget;
    fHost.ready = false;
    fStats = tl_factor_stats{};
    fMean = 0.0f;
    if (!factorPerSm) {
      TL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&factorPerSm, kPcgFactor<S>, TILE, 0));
      if (factorPerSm < 1) throw StatusError{TL_ERR_UNSUPPORTED, "the factored PCG grid cannot be resident"};
    }
  }
  void factorStats(tl_factor_stats* out) override {
    *out = fStats;
    out->mean_iterations = double(fMean);
    out->rows = 3u * fHost.nodes;
    out->ready = fHost.ready ? 1u : 0u;
    out->system_nonzeros = fHost.systemNonZeros;
    out->factor_nonzeros = fHost.factorNonZeros();
  }
  FactorDev factorView() {
    FactorDev f;
    f.nodes = fHost.nodes;
    f.perm = dfPerm.ptr;
    f.iperm = dfIperm.ptr;
    f.row_start = dfRowStart.ptr;
    f.row_col = dfRowCol.ptr;
    f.row_blk = dfRowBlk.ptr;
    f.col_start = dfColStart.ptr;
    f.col_row = dfColRow.ptr;
    f.col_blk = dfColBlk.ptr;
    f.diag_inv = dfDiagInv.ptr;
    f.supernodes = uint32_t(fHost.snParent.size());
    f.sn_start = dfSnStart.ptr;
    f.sn_child = dfSnChild.ptr;
    f.sn_parent = dfSnParent.ptr;
    f.row_split = dfRowSplit.ptr;
    f.col_split = dfColSplit.ptr;
    f.rhs = dfRhs.ptr;
    f.y = dfY.ptr;
    f.w = dfW.ptr;
    f.fwd_flag = dfFlags.ptr;
    f.bwd_flag = dfFlags.ptr + fHost.snParent.size();
    f.ticket = dfTicket.ptr;
    f.epoch = dfTicket.ptr + 3;
    f.frame = dfFrame.ptr;
    f.part = dfPart.ptr;
    return f;
  }
  double fCurStep = 0.0, fCurInertia = 1.0;  // the current step's h and (1 - alpha_m)
  double fCurDamping = 0.0, fDamping = 0.0;   // the current step's damping scale, the factor's
  uint32_t fCgLimit = 0u;                     // Settings::cgIterations of the current step

  // refreshFactor (factor.cc:567-618) for body 0: the system at the rotations
  // of the last element pass, with the damping blocks at the body's positions
  // when a material damps, factored; the FactorReference positions and
  // centre are the body's now.
  void factorRefresh(double step, double inertia, double damping) {
    const auto t0 = std::chrono::steady_clock::now();
    const BodyDev& bd = bodyHost[0];
    const HostBody& h = hb[0];
    const uint32_t V = h.nodes, T = h.tets;
    std::vector<double> rot(size_t(9) * T), x(size_t(3) * V);
    fetchElems<double>(bd, h, rot.data(), nullptr, false);
    getElems<double>(h, rot.data(), nullptr);
    getNodes(bd, h, u, x.data(), true);
    if (!fHost.analyzed || fHost.nodes != V) {  // analyzeSystem (factor.cc:549-565), once per mesh
      fHost.analyze(V, fAnch.data(), fTets, h.rest.data());
      auto put = [&](DevBuf<uint32_t>& d, const std::vector<uint32_t>& v) {
        d.alloc(std::max<size_t>(v.size(), 1));
        d.upload(v.data(), v.size(), st);
      };
      put(dfPerm, fHost.perm);
      put(dfIperm, fHost.iperm);
      put(dfRowStart, fHost.rowStart);
      put(dfRowCol, fHost.rowCol);
      put(dfColStart, fHost.colStart);
      put(dfColRow, fHost.colRow);
      put(dfSnStart, fHost.snStart);
      put(dfRowSplit, fHost.rowSplit);
      put(dfColSplit, fHost.colSplit);
      auto puti = [&](DevBuf<int32_t>& d, const std::vector<int32_t>& v) {
        d.alloc(std::max<size_t>(v.size(), 1));
        d.upload(v.data(), v.size(), st);
      };
      puti(dfSnChild, fHost.snChild);
      puti(dfSnParent, fHost.snParent);
      dfRowBlk.alloc(std::max<size_t>(size_t(9) * fHost.rowCol.size(), 1));
      dfColBlk.alloc(std::max<size_t>(size_t(9) * fHost.rowCol.size(), 1));
      dfDiagInv.alloc(size_t(9) * std::max<uint32_t>(V, 1));
      dfY.alloc(std::max<uint32_t>(V, 1));
      dfW.alloc(std::max<uint32_t>(V, 1));
      dfRhs.alloc(std::max<uint32_t>(V, 1));
      dfFlags.alloc(size_t(2) * std::max<size_t>(fHost.snParent.size(), 1));
      dfFlags.zero(st);
      dfTicket.alloc(4);
      dfTicket.zero(st);
      dfFrame.alloc(9);
      dfPart.alloc(size_t(8) * factorPerSm * ctx->sms);
      dfRef.alloc(size_t(V) + 1);
      for (DevBuf<Vec4<S>>* b : {&dfR, &dfD, &dfQ, &dfZ, &dfRestart}) {
        b->alloc(Vp);
        b->zero(st);
      }
    }
    std::vector<double> blocks(size_t(144) * T), diag(size_t(9) * V, 0.0);
    parallelFor(T, [&](size_t e0, size_t e1) {
      for (size_t e = e0; e < e1; ++e) {
        factorTetBlocks(h.rest.data(), &fTets[4 * e], fYoungs[e], fPoisson[e], &rot[9 * e], step, &blocks[144 * e]);
        const double weight = damping * double(S(fTau[e]));
        if (weight == 0.0) continue;
        double corners[12], d[144];
        for (int c = 0; c < 4; ++c)
          for (int r = 0; r < 3; ++r) corners[3 * c + r] = x[3 * size_t(fTets[4 * e + c]) + r];
        factorDampingBlocks(corners, &rot[9 * e], &fDm[9 * e], fVol[e], fYoungs[e], fPoisson[e], d);
        for (int q = 0; q < 144; ++q) blocks[144 * e + q] += weight * d[q];
      }
    });
    for (uint32_t v = 0; v < V; ++v) {
      const double d = fAnch[v] ? 1.0 : inertia * double(S(fMass[v]));
      diag[9 * size_t(v)] = diag[9 * size_t(v) + 4] = diag[9 * size_t(v) + 8] = d;
    }
    if (fHost.factor(fAnch.data(), fTets, blocks, diag)) {
      dfRowBlk.upload(fHost.rowBlk.data(), fHost.rowBlk.size(), st);
      dfColBlk.upload(fHost.colBlk.data(), fHost.colBlk.size(), st);
      dfDiagInv.upload(fHost.diagInv.data(), fHost.diagInv.size(), st);
    }
    ++fStats.generation;
    fStep = step;
    fInertia = inertia;
    fDamping = damping;
    std::vector<Vec4<double>> ref(size_t(V) + 1);
    double total = 0.0, c[3] = {0.0, 0.0, 0.0};
    for (uint32_t v = 0; v < V; ++v) {
      ref[v] = Vec4<double>{x[3 * size_t(v)], x[3 * size_t(v) + 1], x[3 * size_t(v) + 2], 0.0};
      const double m = double(S(fMass[v]));
      total += m;
      for (int k = 0; k < 3; ++k) c[k] += m * x[3 * size_t(v) + k];
    }
    ref[V] = total > 0.0 ? Vec4<double>{c[0] / total, c[1] / total, c[2] / total, 0.0}
                         : Vec4<double>{c[0], c[1], c[2], 0.0};
    dfRef.upload(ref.data(), ref.size(), st);
    TL_CUDA(cudaStreamSynchronize(st));
    fStats.refactor_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }

  // One kPcgFactor solve from X (or zero) with the given cap; its result.
  CgBodyDev launchFactor(Vec4<S>* X, bool x0zero, uint32_t limit, uint32_t pass) {
    kPcgPrepare<S><<<1, TILE, 0, st>>>(view(), pass);
    check();
    Sys<S> s = view();
    SellDev<S> g = sellView();
    FactorDev f = factorView();
    Vec4<S>*R = dfR.ptr, *D = dfD.ptr, *Q = dfQ.ptr, *Z = dfZ.ptr;
    uint32_t xz = x0zero ? 1u : 0u, lim = limit;
    void* args[] = {&s, &g, &f, &X, &R, &D, &Q, &Z, &xz, &lim};
    TL_CUDA(cudaLaunchCooperativeKernel((const void*)kPcgFactor<S>, dim3(factorPerSm * ctx->sms), dim3(TILE), args,
                                        0, st));
    ++launches;
    CgBodyDev c;
    TL_CUDA(cudaMemcpyAsync(&c, cg.ptr, sizeof(CgBodyDev), cudaMemcpyDeviceToHost, st));
    TL_CUDA(cudaStreamSynchronize(st));
    return c;
  }

  // solvePrimary (solver.cc:3822-3910) with a prepared factor.  The solves
  // that may refresh (a substep's first elastic read, a Newton attempt's
  // first solve, a fallback's first read) are exactly those that start from
  // a guess; a capped one makes the factor again at the latest rotations and
  // solves again from the same start with the full iteration cap.
  void pcgFactor(int law, Vec4<S>* X, uint32_t pass, bool x0zero, bool tangent) {
    const bool refreshes = !x0zero;
    Sys<S> s = view();
    SellDev<S> g = sellView();
    const unsigned blocks = (sellUpperCount + TILE - 1) / TILE;
    if (profiling) mark(1, true);
    assembleSell(s, g, blocks, law == TL_LAW_SNH ? 1 : 0, hasDamping && law != TL_LAW_SNH, tangent, pass);
    check();
    ++launches;
    if (profiling) {
      mark(1, false);
      mark(2, true);
    }
    if (refreshes)
      TL_CUDA(cudaMemcpyAsync(dfRestart.ptr, X, size_t(Vp) * sizeof(Vec4<S>), cudaMemcpyDeviceToDevice, st));
    CgBodyDev c = launchFactor(X, x0zero, fBudget, pass);
    if (c.pad0 && refreshes) {
      ++fStats.refresh_requests;
      fStats.refreshed_at_age = fStats.substeps_since_refresh;
      fStats.spent_before_refresh = c.taken;
      fStats.wasted_iterations += c.taken;
      fStats.refresh_requested = 1u;
      TL_CUDA(cudaMemcpyAsync(X, dfRestart.ptr, size_t(Vp) * sizeof(Vec4<S>), cudaMemcpyDeviceToDevice, st));
      factorRefresh(fCurStep, fCurInertia, fCurDamping);
      ++fStats.refactors;
      ++fStats.retries;
      ++fStats.refactor_count;
      ++fStats.retry_count;
      fStats.factor_age = 0u;
      fStats.substeps_since_refresh = 0u;
      identityFrame();
      if (fHost.ready) {
        c = launchFactor(X, x0zero, fCgLimit, pass);
      } else {  // an empty factor conditions by block Jacobi (solver.cc:1923-1944)
        if (profiling) mark(2, false);
        fPrepared = false;
        pcg(law, X, pass, x0zero, tangent);
        fPrepared = true;
        TL_CUDA(cudaMemcpyAsync(&c, cg.ptr, sizeof(CgBodyDev), cudaMemcpyDeviceToHost, st));
        TL_CUDA(cudaStreamSynchronize(st));
        fStats.spent_after_refresh = c.taken;
        if (c.taken == fCgLimit && std::sqrt(c.length) > c.target) {
          ++fStats.retries_failed;
          fStats.fresh_retry_failed = 1u;
        }
        return;
      }
      fStats.spent_after_refresh = c.taken;
      if (c.pad0) {
        ++fStats.retries_failed;
        fStats.fresh_retry_failed = 1u;
      }
    }
    fStats.factor_applications += c.pad1;
    kFactorRecord<S><<<1, 1, 0, st>>>(view(), tangent ? 1u : 0u);
    check();
    if (profiling) mark(2, false);
    if (tracing) trace.push_back(c.taken);
  }

  void identityFrame() {
    const double eye[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    dfFrame.upload(eye, 9, st);
    TL_CUDA(cudaStreamSynchronize(st));
  }
  void finalize(uint32_t which) {
    kFinalize<<<B, TILE, 0, st>>>(dBody.ptr, epart.ptr, npart.ptr, acc.ptr, which);
    check();
  }
  void nodeOp(void (*k)(Sys<S>, uint32_t), uint32_t pass) {
    k<<<nodeTiles, TILE, 0, st>>>(view(), pass);
    check();
  }
  void copy(DevBuf<Vec4<S>>& dst, const DevBuf<Vec4<S>>& src) {
    TL_CUDA(cudaMemcpyAsync(dst.ptr, src.ptr, size_t(Vp) * sizeof(Vec4<S>), cudaMemcpyDeviceToDevice, st));
  }
  BodyAccDev readAcc(uint32_t b) {
    BodyAccDev* h = hAcc.get(B);
    acc.download(h, B, st);
    TL_CUDA(cudaStreamSynchronize(st));
    return h[b];
  }
  uint32_t readCount(DevBuf<uint32_t>& buf, uint32_t b) {
    uint32_t* h = hCount.get(B);
    buf.download(h, B, st);
    TL_CUDA(cudaStreamSynchronize(st));
    return h[b];
  }

  // -------------------------------------------------------------- step ----

  int32_t step(const tl_settings& set, const double gvec[3], double dt, tl_step_report* reports) override {
    if (set.law > 1u) throw StatusError{TL_ERR_ARG, "unknown law"};
    if (hasDamping && set.law == TL_LAW_SNH)
      throw StatusError{TL_ERR_UNSUPPORTED, "stiffness damping is defined with the corotated law"};
    if (hencky && (set.law != TL_LAW_COROTATED || hasDamping))
      throw StatusError{TL_ERR_UNSUPPORTED, "the finite-strain flow is written for the corotated law without damping"};
    const int law = int(set.law);
    if (set.rigid_split > TL_RIGID_SPLIT_PROJECTED) throw StatusError{TL_ERR_ARG, "unknown rigid split"};
    bool anyFloating = false;
    for (uint32_t b = 0; b < B; ++b) {
      if (!hb[b].floats(set.rigid_split)) continue;
      if (!(hb[b].mass > 0.0)) throw StatusError{TL_ERR_ARG, "a floating body needs a positive total mass"};
      anyFloating = true;
    }
    if (anyFloating) ensureFloating();
    launches = 0;
    solveCount = 0;
    profiling = (set.flags & TL_FLAG_PROFILE) != 0u;
    tracing = (set.flags & TL_FLAG_TRACE) != 0u;
    evUsed.clear();
    // the barrier error word is cleared once per step; a wait that runs out in
    // any of the step's solves is reported when the step ends
    TL_CUDA(cudaMemsetAsync(&sync.ptr->error, 0, sizeof(int), st));
    {
      const bool yieldsLaw = law == TL_LAW_COROTATED && !hencky &&
                             std::any_of(hb.begin(), hb.end(), [](const HostBody& h) { return h.anyYields; });
      const bool newtonNeeded = set.plastic_passes > 1u && yieldsLaw;
      if (B > 1 && !newtonNeeded && tuneGraph && !graphBroken && !tracing && !hencky && expireSolve < 0) {
        const int32_t rc = stepGraph(set, gvec, dt, reports, law, yieldsLaw, anyFloating);
        if (rc != TL_ERR_UNSUPPORTED) return rc;  // unsupported: capture refused, fall through to launches
      }
    }
    cudaEvent_t e0, e1;
    TL_CUDA(cudaEventCreate(&e0));
    TL_CUDA(cudaEventCreate(&e1));
    TL_CUDA(cudaEventRecord(e0, st));
    const uint32_t configured = std::max(set.substeps, 1u);
    const Rule rule = ruleOf(set.spectral_radius);
    const double checkInner = dt / double(configured);
    // ---- per-body constants and the predictor-inversion test (solver.cc:3574-3583)
    BodyStepDev* hs = hStep.get(B);
    for (uint32_t b = 0; b < B; ++b) {
      BodyStepDev& s = hs[b];
      std::memset(&s, 0, sizeof(s));
      s.substeps = configured;
      s.limit = set.cg_iterations;
      s.alpha_f = rule.alphaForce;
      s.alpha_m = rule.alphaMass;
      s.beta = rule.beta;
      s.gamma = rule.gamma;
      s.gx = gvec[0];
      s.gy = gvec[1];
      s.gz = gvec[2];
      s.floating = hb[b].floats(set.rigid_split) ? 1u : 0u;
      s.projected = set.rigid_split == TL_RIGID_SPLIT_PROJECTED ? 1u : 0u;
      // a floating body solves to at most FLOATING_TOLERANCE (solver.cc:3560-3562)
      s.tolerance = s.floating ? std::min(set.tolerance, FLOATING_TOLERANCE) : set.tolerance;
      s.check_inner = checkInner;
      s.check_carry = (0.5 - rule.beta) * checkInner * checkInner;
    }
    dStep.upload(hs, B, st);
    {
      BodyAccDev* h = hAcc.get(B);
      for (uint32_t b = 0; b < B; ++b) {
        std::memset(&h[b], 0, sizeof(BodyAccDev));
        h[b].min_j_key = ~0ull;
      }
      acc.upload(h, B, st);
      cgrep.zero(st);
    }
    kInversionCheck<S><<<elemTiles, TILE, 0, st>>>(view());
    check();
    ++launches;
    BodyAccDev* ha = hAcc.get(B);
    acc.download(ha, B, st);
    TL_CUDA(cudaStreamSynchronize(st));
    uint32_t maxSub = 1;
    bool anyNewton = false;
    std::vector<uint8_t> newtonBody(B, 0u);
    for (uint32_t b = 0; b < B; ++b) {
      BodyStepDev& s = hs[b];
      s.substeps = ha[b].inverts ? std::max(configured, INVERTED_SUBSTEPS) : configured;
      s.inner = dt / double(s.substeps);
      s.carry = (0.5 - rule.beta) * s.inner * s.inner;
      s.inertia = 1.0 - rule.alphaMass;
      s.hstep = std::sqrt((1.0 - rule.alphaForce) * rule.beta) * s.inner;
      s.scale = s.hstep * s.hstep;
      maxSub = std::max(maxSub, s.substeps);
      const bool yieldsHere = hb[b].anyYields && law == TL_LAW_COROTATED && !hencky;
      newtonBody[b] = (set.plastic_passes > 1u && yieldsHere) ? 1u : 0u;
      anyNewton = anyNewton || newtonBody[b];
    }
    dStep.upload(hs, B, st);
    const bool anyYields = std::any_of(hb.begin(), hb.end(), [](const HostBody& h) { return h.anyYields; }) &&
                           law == TL_LAW_COROTATED && !hencky;
    std::vector<tl_step_report> local(B);
    fPrepared = false;
    if (factorOn) {
      if (B != 1 || hencky)
        throw StatusError{TL_ERR_UNSUPPORTED, "a solver state needs one body on the small-strain path"};
      // the factor is made at the committed rotations, which the SNH operator state replaces
      if (law == TL_LAW_SNH) throw StatusError{TL_ERR_UNSUPPORTED, "a solver state is held for the corotated law"};
      // solver.cc:3639-3655: the factor is made again when it is empty or was
      // made for another step or inertia
      fCurStep = hs[0].hstep;
      fCurInertia = hs[0].inertia;
      // dampingStep (solver.cc:3592): (1 - alpha_f) gamma h when a material damps
      fCurDamping = hasDamping ? (1.0 - rule.alphaForce) * rule.gamma * hs[0].inner : 0.0;
      fCgLimit = set.cg_iterations;
      if (!fHost.ready || fStep != fCurStep || fInertia != fCurInertia || fDamping != fCurDamping) {
        factorRefresh(fCurStep, fCurInertia, fCurDamping);
        fStats.factor_age = 0u;
        ++fStats.refactor_count;
      }
    }
    for (uint32_t pass = 0; pass < maxSub; ++pass) {
      if (factorOn) {  // solver.cc:3808-3821: the prepared factor, its frame and budget
        fPrepared = fHost.ready;
        if (fPrepared) {
          kFactorFrame<S><<<1, TILE, 0, st>>>(view(), hb[0].nodes, dfRef.ptr, dfFrame.ptr);
          check();
        }
        fBudget = fPrepared && factorBudget != 0u ? std::min(factorBudget, set.cg_iterations) : set.cg_iterations;
      }
      if (anyFloating) frameBegin(pass);
      nodeOp(kPredict<S>, pass);
      if (!anyNewton) {
        elasticReads(law, pass);
      } else if (B == 1u) {
        newton(law, pass, set, rule, hs[0], local[0]);
      } else {  // a batch: every yielding body's Newton loop at once, the others' elastic reads
        newtonBatch(law, pass, set, rule, hs, local, newtonBody);
      }
      if (factorOn) {  // solver.cc:4258-4263
        CgReportDev rep;
        TL_CUDA(cudaMemcpyAsync(&rep, cgrep.ptr, sizeof(CgReportDev), cudaMemcpyDeviceToHost, st));
        TL_CUDA(cudaStreamSynchronize(st));
        ++fStats.substeps_since_refresh;
        fMean = 0.9f * fMean + 0.1f * float(rep.pass_iterations);
      }
      if (anyFloating) frameEnd(pass);
      nodeOp(kUpdate<S>, pass);
      if (anyFloating) frameTurn(pass);
      recordSubstep(pass);
      if (anyYields) element(law, u.ptr, nullptr, pass, EM_MAPPING | EM_COMMIT, 0.0);
    }
    fPrepared = false;
    if (hencky) {  // flowLattice once per step, after the solve (strainstep.cc:822-825)
      yielding.zero(st);
      kHenckyFlow<S><<<elemTiles, TILE, 0, st>>>(view());
      check();
    }
    kStepEnd<S><<<nodeTiles, TILE, 0, st>>>(view());
    check();
    finalize(0);
    finalize(2);
    TL_CUDA(cudaEventRecord(e1, st));
    BodyAccDev* hacc = hAcc.get(B);
    acc.download(hacc, B, st);
    CgReportDev* hrep = hRep.get(B);
    cgrep.download(hrep, B, st);
    GridSyncDev* hsy = hSync.get(1);
    sync.download(hsy, 1, st);
    uint32_t* hy = hCount.get(B);
    yielding.download(hy, B, st);
    subrec.download(hSubrec.get(size_t(B) * SUBSTEP_RECORDS), size_t(B) * SUBSTEP_RECORDS, st);
    TL_CUDA(cudaStreamSynchronize(st));
    {
      std::vector<uint32_t> counts(B);
      for (uint32_t b = 0; b < B; ++b) counts[b] = hs[b].substeps;
      keepSubsteps(counts.data());
    }
    float ms = 0.f;
    TL_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    double classSeconds[3] = {0.0, 0.0, 0.0};
    for (const auto& u : evUsed) {
      float t = 0.f;
      TL_CUDA(cudaEventElapsedTime(&t, evPool[u.second].first, evPool[u.second].second));
      classSeconds[u.first] += double(t) * 1e-3;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int32_t status = TL_OK;
    if (hsy->error != 0) {
      if (dfFlags.ptr) {  // a factored solve may have left mid-application: its flags start over
        dfFlags.zero(st);
        dfTicket.zero(st);
        TL_CUDA(cudaStreamSynchronize(st));
      }
      throw StatusError{TL_ERR_TIMEOUT, "a PCG grid barrier ran out of time"};
    }
    for (uint32_t b = 0; b < B; ++b) {
      if (!reports) continue;
      tl_step_report& r = reports[b];
      const tl_step_report& l = local[b];
      r.nodes += hb[b].nodes;
      r.elements += hb[b].tets;
      r.substeps += hs[b].substeps;
      r.cg_iterations += hrep[b].iterations;
      r.cg_capped_solves += hrep[b].capped;
      r.operator_applications += hrep[b].applications;
      r.cg_worst_relative_residual = std::max(r.cg_worst_relative_residual, hrep[b].worst_rel);
      r.plastic_evaluations += l.plastic_evaluations;
      r.plastic_solves += l.plastic_solves;
      r.plastic_backtracks += l.plastic_backtracks;
      r.plastic_capped += l.plastic_capped;
      r.plastic_linear_reads += l.plastic_linear_reads;
      r.plastic_handoffs += l.plastic_handoffs;
      r.plastic_fallbacks += l.plastic_fallbacks;
      r.plastic_fallback_rejections += l.plastic_fallback_rejections;
      r.plastic_worst_residual = std::max(r.plastic_worst_residual, l.plastic_worst_residual);
      r.yielding = (B > 1u && newtonBody[b]) ? l.yielding : hy[b];
      r.plastic_growth |= hacc[b].grew;
      r.non_finite |= hacc[b].nonfinite;
      r.elastic_energy += hacc[b].energy;
      r.kinetic_energy += hacc[b].kinetic;
      r.min_volume_ratio = fromMinKey(hacc[b].min_j_key);
      r.device_seconds += double(ms) * 1e-3;
      r.kernel_launches += launches;
      r.cg_tangent_iterations += hrep[b].tangent_iterations;
      r.cg_solves += hrep[b].solves;
      r.element_seconds += classSeconds[0];
      r.assemble_seconds += classSeconds[1];
      r.pcg_seconds += classSeconds[2];
    }
    for (uint32_t b = 0; b < B; ++b)
      if (hacc[b].nonfinite) status = TL_ERR_NONFINITE;
    return status;
  }

  // ------------------------------------------------- graph-captured step ----
  // A batched elastic step as one fixed launch sequence: the predictor
  // inversion test and the substep count are decided on the device
  // (kStepSelect), every body runs max(configured, 4) passes with the passes
  // beyond its own substep count masked off, and the whole sequence is
  // captured once into a CUDA graph and replayed every step.  The constants
  // are copied from pinned host memory by a graph node, so dt and gravity may
  // change between steps without re-capturing.
  cudaGraphExec_t graphExec = nullptr;
  uint64_t graphKey = ~0ull;
  bool graphBroken = false;
  DevBuf<BodyStepDev> dStepVar;
  PinnedBuf<BodyStepDev> hStepVar, hStepOut;

  // The step's opening, launched directly: the constants, the accumulators,
  // the predictor-inversion test and each body's substep choice, whose
  // largest count is read back to pick the graph.
  uint32_t openStep() {
    TL_CUDA(cudaMemcpyAsync(dStepVar.ptr, hStepVar.ptr, sizeof(BodyStepDev) * 2 * B, cudaMemcpyHostToDevice, st));
    const uint32_t bb = (B + 255) / 256;
    TL_CUDA(cudaMemsetAsync(&sync.ptr->error, 0, sizeof(int), st));
    kAccReset<<<bb, 256, 0, st>>>(acc.ptr, cgrep.ptr, B);
    kStepSelect<<<bb, 256, 0, st>>>(dStep.ptr, dStepVar.ptr, acc.ptr, B, 0u);
    kInversionCheck<S><<<elemTiles, TILE, 0, st>>>(view());
    kStepSelect<<<bb, 256, 0, st>>>(dStep.ptr, dStepVar.ptr, acc.ptr, B, 1u);
    TL_CUDA(cudaGetLastError());
    dStep.download(hStepOut.ptr, B, st);
    TL_CUDA(cudaStreamSynchronize(st));
    uint32_t passes = 1;
    for (uint32_t b = 0; b < B; ++b) passes = std::max(passes, hStepOut.ptr[b].substeps);
    return passes;
  }
  // The captured part: `passes` substeps (bodies with fewer are masked off in
  // the later ones), the step's end and the downloads of its results.
  void enqueueStep(int law, uint32_t passes, bool yieldsLaw, bool anyFloating) {
    for (uint32_t pass = 0; pass < passes; ++pass) {
      if (anyFloating) frameBegin(pass);
      nodeOp(kPredict<S>, pass);
      elasticReads(law, pass);
      if (anyFloating) frameEnd(pass);
      nodeOp(kUpdate<S>, pass);
      if (anyFloating) frameTurn(pass);
      recordSubstep(pass);
      if (yieldsLaw) element(law, u.ptr, nullptr, pass, EM_MAPPING | EM_COMMIT, 0.0);
    }
    kStepEnd<S><<<nodeTiles, TILE, 0, st>>>(view());
    finalize(0);
    finalize(2);
    acc.download(hAcc.ptr, B, st);
    cgrep.download(hRep.ptr, B, st);
    sync.download(hSync.ptr, 1, st);
    yielding.download(hCount.ptr, B, st);
    dStep.download(hStepOut.ptr, B, st);
    subrec.download(hSubrec.ptr, size_t(B) * SUBSTEP_RECORDS, st);
  }

  int32_t stepGraph(const tl_settings& set, const double gvec[3], double dt, tl_step_report* reports, int law,
                    bool yieldsLaw, bool anyFloating) {
    const uint32_t configured = std::max(set.substeps, 1u);
    const Rule rule = ruleOf(set.spectral_radius);
    if (!dStepVar.ptr) dStepVar.alloc(size_t(2) * B);
    BodyStepDev* hv = hStepVar.get(size_t(2) * B);
    hAcc.get(B);
    hRep.get(B);
    hSync.get(1);
    hCount.get(B);
    hStepOut.get(B);
    hSubrec.get(size_t(B) * SUBSTEP_RECORDS);
    for (uint32_t b = 0; b < B; ++b)
      for (uint32_t k = 0; k < 2; ++k) {
        BodyStepDev& s = hv[2 * b + k];
        std::memset(&s, 0, sizeof(s));
        s.substeps = k == 0 ? configured : std::max(configured, INVERTED_SUBSTEPS);
        s.limit = set.cg_iterations;
        s.alpha_f = rule.alphaForce;
        s.alpha_m = rule.alphaMass;
        s.beta = rule.beta;
        s.gamma = rule.gamma;
        s.gx = gvec[0];
        s.gy = gvec[1];
        s.gz = gvec[2];
        s.floating = hb[b].floats(set.rigid_split) ? 1u : 0u;
        s.projected = set.rigid_split == TL_RIGID_SPLIT_PROJECTED ? 1u : 0u;
        s.tolerance = s.floating ? std::min(set.tolerance, FLOATING_TOLERANCE) : set.tolerance;
        s.check_inner = dt / double(configured);
        s.check_carry = (0.5 - rule.beta) * s.check_inner * s.check_inner;
        s.inner = dt / double(s.substeps);
        s.carry = (0.5 - rule.beta) * s.inner * s.inner;
        s.inertia = 1.0 - rule.alphaMass;
        s.hstep = std::sqrt((1.0 - rule.alphaForce) * rule.beta) * s.inner;
        s.scale = s.hstep * s.hstep;
      }
    cudaEvent_t e0, e1;
    TL_CUDA(cudaEventCreate(&e0));
    TL_CUDA(cudaEventCreate(&e1));
    TL_CUDA(cudaEventRecord(e0, st));
    const uint32_t passes = openStep();
    // one graph per substep count (the configured count, or the inverted
    // predictor's four), so a step replays exactly the passes it takes
    const uint64_t key = (uint64_t(law) << 48) | (uint64_t(yieldsLaw) << 40) | (uint64_t(anyFloating) << 38) |
                         (uint64_t(profiling) << 36) | (uint64_t(passes) << 24) | (uint64_t(configured) << 8) |
                         uint64_t(tuneBlocksPerSm & 0xffu);
    if (!graphExec || graphKey != key) {
      if (graphExec) cudaGraphExecDestroy(graphExec);
      graphExec = nullptr;
      cudaGraph_t graph = nullptr;
      evUsed.clear();  // profiling marks become event-record nodes of the graph
      TL_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
      launches = 0;
      capturing = true;
      try {
        enqueueStep(law, passes, yieldsLaw, anyFloating);
      } catch (...) {
        capturing = false;
        cudaStreamEndCapture(st, &graph);
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        graphBroken = true;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return TL_ERR_UNSUPPORTED;
      }
      capturing = false;
      const cudaError_t ended = cudaStreamEndCapture(st, &graph);
      if (ended != cudaSuccess || !graph ||
          cudaGraphInstantiate(&graphExec, graph, 0) != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        graphExec = nullptr;
        graphBroken = true;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return TL_ERR_UNSUPPORTED;
      }
      cudaGraphDestroy(graph);
      graphKey = key;
      graphLaunches = launches;
      graphEv = evUsed;
    }
    TL_CUDA(cudaGraphLaunch(graphExec, st));
    TL_CUDA(cudaEventRecord(e1, st));
    TL_CUDA(cudaStreamSynchronize(st));
    float ms = 0.f;
    TL_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    double classSeconds[3] = {0.0, 0.0, 0.0};
    if (profiling)
      for (const auto& u : graphEv) {
        float t = 0.f;
        TL_CUDA(cudaEventElapsedTime(&t, evPool[u.second].first, evPool[u.second].second));
        classSeconds[u.first] += double(t) * 1e-3;
      }
    if (hSync.ptr->error != 0) throw StatusError{TL_ERR_TIMEOUT, "a PCG grid barrier ran out of time"};
    {
      std::vector<uint32_t> counts(B);
      for (uint32_t b = 0; b < B; ++b) counts[b] = hStepOut.ptr[b].substeps;
      keepSubsteps(counts.data());
    }
    int32_t status = TL_OK;
    for (uint32_t b = 0; b < B; ++b) {
      if (hAcc.ptr[b].nonfinite) status = TL_ERR_NONFINITE;
      if (reports) {
        reports[b].element_seconds += classSeconds[0];
        reports[b].assemble_seconds += classSeconds[1];
        reports[b].pcg_seconds += classSeconds[2];
      }
      if (!reports) continue;
      tl_step_report& r = reports[b];
      r.nodes += hb[b].nodes;
      r.elements += hb[b].tets;
      r.substeps += hStepOut.ptr[b].substeps;
      r.cg_iterations += hRep.ptr[b].iterations;
      r.cg_capped_solves += hRep.ptr[b].capped;
      r.operator_applications += hRep.ptr[b].applications;
      r.cg_solves += hRep.ptr[b].solves;
      r.cg_tangent_iterations += hRep.ptr[b].tangent_iterations;
      r.cg_worst_relative_residual = std::max(r.cg_worst_relative_residual, hRep.ptr[b].worst_rel);
      r.yielding = hCount.ptr[b];
      r.plastic_growth |= hAcc.ptr[b].grew;
      r.non_finite |= hAcc.ptr[b].nonfinite;
      r.elastic_energy += hAcc.ptr[b].energy;
      r.kinetic_energy += hAcc.ptr[b].kinetic;
      r.min_volume_ratio = fromMinKey(hAcc.ptr[b].min_j_key);
      r.device_seconds += double(ms) * 1e-3;
      r.kernel_launches += graphLaunches + OPEN_LAUNCHES;
    }
    return status;
  }
  uint32_t graphLaunches = 0;
  static constexpr uint32_t OPEN_LAUNCHES = 4;  // openStep's kernels
  std::vector<std::pair<int, size_t>> graphEv;  // event pairs recorded by the captured graph

  void setSolver(uint32_t form) override { solverForm = form; }
  void expireWait(int32_t solve) override { expireSolve = solve; }
  void setFlowLimits(uint32_t b, uint32_t lane, double crushStress, double crushLimit, double plasticMax) override {
    if (b >= B || lane >= hb[b].lanes) throw StatusError{TL_ERR_ARG, "no such body or material lane"};
    const size_t at = size_t(3) * (hb[b].laneBase + lane);
    hFlim[at] = crushStress;
    hFlim[at + 1] = crushLimit;
    hFlim[at + 2] = plasticMax;
    dFlim.upload(hFlim.data() + at, 3, st, at);
    TL_CUDA(cudaStreamSynchronize(st));
  }
  // Does a step under `law` read or write the plastic slot?
  bool plasticUsed(uint32_t law) const override {
    if (hencky) return true;
    return law == TL_LAW_COROTATED &&
           std::any_of(hb.begin(), hb.end(), [](const HostBody& h) { return h.anyYields; });
  }
  // Every tet starts from its authored rest: P = I, hardening 0.
  void setPlasticity(uint32_t mode) override {
    if (mode != TL_PLASTICITY_HENCKY) {
      hencky = false;
      return;
    }
    if (!hk.ptr) hk.alloc(size_t(10) * Tp);
    std::vector<double> h(size_t(10) * Tp, 0.0);
    std::fill(h.begin(), h.begin() + Tp, 1.0);
    std::fill(h.begin() + size_t(4) * Tp, h.begin() + size_t(5) * Tp, 1.0);
    std::fill(h.begin() + size_t(8) * Tp, h.begin() + size_t(9) * Tp, 1.0);
    hk.upload(h.data(), h.size(), st);
    TL_CUDA(cudaStreamSynchronize(st));
    hencky = true;
  }
  void tune(uint32_t blocksPerSm, uint32_t graph) override {
    tuneBlocksPerSm = blocksPerSm;
    tuneGraph = graph != 0u;
    if (graphExec) cudaGraphExecDestroy(graphExec);
    graphExec = nullptr;
    graphBroken = false;
  }
  void tuneShape(uint32_t knob, uint32_t value) override {
    if (knob == TL_SHAPE_ROW_GROUP) {
      if (value != 0u && value != 2u && value != 4u) throw StatusError{TL_ERR_ARG, "row group is 0, 2 or 4"};
      tuneRowGroup = value;
    } else if (knob == TL_SHAPE_BATCH_BLOCKS) {
      if (value != 0u && value != 3u && value != 4u) throw StatusError{TL_ERR_ARG, "batch blocks per SM are 0, 3 or 4"};
      tuneBatchBlocks = value;
    } else {
      throw StatusError{TL_ERR_ARG, "no such launch-shape knob"};
    }
    if (sellReady) {
      sellPerSm = sellPerSmOf[sellU() == 4u ? 1 : 0];
      batchSellPerSm = occupancyOf(batchKernel(true), 0);
      batchPipePerSm = occupancyOf(batchKernel(false), 0);
      if (batchSellPerSm < 1 || batchPipePerSm < 1) throw StatusError{TL_ERR_CUDA, "shape cannot be resident"};
    }
    if (graphExec) cudaGraphExecDestroy(graphExec);  // the captured launches hold the old kernels
    graphExec = nullptr;
  }

  // solver.cc:3914-3950: assemble at the predictor, solve for the
  // acceleration, then two re-linearised increments.
  // newtonReads is ANCHORED_READS except inside a differentiable rollout.
  uint32_t newtonReads = ANCHORED_READS;
  void elasticReads(int law, uint32_t pass) {
    element(law, weighted.ptr, nullptr, pass, EM_MAPPING, 0.0);
    nodeAssemble(nullptr, pass);
    pcg(law, a.ptr, pass, false, false);
    for (uint32_t read = 1; read < newtonReads; ++read) {
      element(law, weighted.ptr, a.ptr, pass, EM_MAPPING, 0.0);
      nodeAssemble(a.ptr, pass);
      pcg(law, incr.ptr, pass, true, false);
      kAddIncrement<S><<<nodeTiles, TILE, 0, st>>>(view(), a.ptr, pass);
      check();
    }
  }

  // The plastic Newton loop of solver.cc:3951-4250 for one body (b = 0).
  void newton(int law, uint32_t pass, const tl_settings& set, const Rule& rule, const BodyStepDev& bs,
              tl_step_report& rep) {
    const double travel = rule.beta * bs.inner * bs.inner;
    const uint32_t plasticCap = set.plastic_passes;
    bool consistent = false;  // bindStiffness(false) at step start (solver.cc:3521)
    auto bind = [&](bool want) { consistent = want; };
    auto assemble = [&](double margin, bool mapping = true) {
      const uint32_t mode = (mapping ? uint32_t(EM_MAPPING) : 0u) | (consistent ? uint32_t(EM_CONSISTENT) : 0u);
      element(law, weighted.ptr, total.ptr, pass, mode, margin);
    };
    // |right|^2 after the node assembly, and the loading count of the element
    // pass before it, read back in one wait
    auto balanceSquared = [&](uint32_t& loadingNow) {
      nodeAssemble(total.ptr, pass);
      finalize(1);
      BodyAccDev* ha = hAcc.get(B);
      uint32_t* hc = hCount.get(B);
      acc.download(ha, B, st);
      loading.download(hc, B, st);
      TL_CUDA(cudaStreamSynchronize(st));
      loadingNow = hc[0];
      return ha[0].right_sq;
    };
    auto solve = [&](bool x0zero) { pcg(law, incr.ptr, pass, x0zero, consistent); };
    auto addToTotal = [&]() {
      kAddIncrement<S><<<nodeTiles, TILE, 0, st>>>(view(), total.ptr, pass);
      check();
    };
    bool linearAllowed = true;
    for (;;) {
      total.zero(st);
      double accepted = std::numeric_limits<double>::infinity();
      double opening = 0.0;
      double lowest = std::numeric_limits<double>::infinity();
      uint32_t loadingBefore = 0, solves = 0;
      bool converged = false, predictorUnloaded = false, handedOff = false;
      for (uint32_t attempt = 0; attempt != plasticCap; ++attempt) {
        if (attempt < 2u) bind(attempt != 0u);
        assemble(LOADING_MARGIN);
        ++rep.plastic_evaluations;
        uint32_t loadingNow = 0;
        const double squared = balanceSquared(loadingNow);
        if (attempt != 0u) {
          const double ranked = std::isfinite(squared) ? squared : std::numeric_limits<double>::infinity();
          if (attempt == 1u || ranked < lowest) {
            lowest = ranked;
            copy(lowest_(), total);
          }
        }
        if (attempt == 0u) predictorUnloaded = loadingNow == 0u;
        if (attempt == 1u && linearAllowed && predictorUnloaded && std::isfinite(squared) && squared > accepted) {
          ++rep.plastic_linear_reads;
          bind(false);
          for (uint32_t read = 1; read != ANCHORED_READS; ++read) {
            assemble(LOADING_MARGIN);
            ++rep.plastic_evaluations;
            if (readCount(loading, 0) != 0u) {
              handedOff = true;
              break;
            }
            nodeAssemble(total.ptr, pass);
            solve(true);
            ++solves;
            addToTotal();
          }
          converged = !handedOff;
          break;
        }
        if (attempt != 0u && !(squared <= accepted)) {
          nodeOp(kBacktrack<S>, pass);
          ++rep.plastic_backtracks;
          continue;
        }
        if (attempt != 0u && loadingBefore == 0u && loadingNow == 0u) {
          converged = true;
          break;
        }
        opening = attempt == 0u ? squared : opening;
        accepted = squared;
        loadingBefore = loadingNow;
        if (attempt == 0u) copy(incr, a);
        solve(attempt != 0u);
        ++solves;
        TL_CUDA(cudaMemsetAsync(&acc.ptr[0].moved_key, 0, 2 * sizeof(unsigned long long), st));
        nodeOp(kNewtonAccept<S>, pass);
        const BodyAccDev h = readAcc(0);
        double moved, extent;
        std::memcpy(&moved, &h.moved_key, 8);
        std::memcpy(&extent, &h.extent_key, 8);
        if (solves > 1u &&
            travel * moved <= PLASTIC_RESOLUTION * double(std::numeric_limits<float>::epsilon()) * extent) {
          converged = true;
          break;
        }
      }
      rep.plastic_solves += solves;
      if (handedOff) {
        ++rep.plastic_handoffs;
        linearAllowed = false;
        continue;
      }
      if (!converged) {
        bind(false);
        total.zero(st);
        bool fellBack = true;
        for (uint32_t read = 0; read != ANCHORED_READS; ++read) {
          assemble(LOADING_MARGIN, read != 0u);
          ++rep.plastic_evaluations;
          if (readCount(loading, 0) != 0u) {
            fellBack = false;
            break;
          }
          nodeAssemble(total.ptr, pass);
          if (read == 0u) copy(incr, a);
          solve(read != 0u);
          ++rep.plastic_solves;
          addToTotal();
        }
        if (fellBack) {
          assemble(LOADING_MARGIN);
          ++rep.plastic_evaluations;
          uint32_t loadingNow = 0;
          const double squared = balanceSquared(loadingNow);
          fellBack = loadingNow == 0u && squared <= PLASTIC_REDUCTION * PLASTIC_REDUCTION * opening;
        }
        if (fellBack) {
          ++rep.plastic_fallbacks;
          converged = true;
        } else {
          ++rep.plastic_fallback_rejections;
          bind(true);
          copy(total, lowest_());
          assemble(LOADING_MARGIN);
          ++rep.plastic_evaluations;
          nodeAssemble(total.ptr, pass);
          const double remaining = std::sqrt(lowest);
          if (remaining >= rep.plastic_worst_residual) rep.plastic_worst_residual = remaining;
        }
      }
      rep.plastic_capped += converged ? 0u : 1u;
      copy(a, total);
      break;
    }
  }
  DevBuf<Vec4<S>>& lowest_() { return lowest; }

  // ------------------------------------------- batched plastic Newton ----
  // The plastic Newton loop of solver.cc:3951-4250 for every yielding body of
  // a batch at once.  Each body runs the single-body control flow of newton()
  // above as a state machine on the host; the device work is issued in
  // rounds, each round one element pass and node assembly for the bodies
  // that want one (gate GATE_ASSEMBLE) and one PCG solve for the bodies that
  // want one (gates GATE_SOLVE0 + group), with per-body masked copies in
  // between.  Every body therefore makes exactly the device calls it makes
  // alone, in the same order; only bodies' calls are grouped.  Each round
  // reads the per-body results back once after the assembly and once after
  // the solves.
  struct NewtonBody {
    enum Stage : uint8_t {
      START, ATTEMPT, ATTEMPT_GOT, ATTEMPT_SOLVED, LINEAR, LINEAR_GOT, LINEAR_SOLVED, AFTER, FALLBACK, FALLBACK_GOT,
      FALLBACK_SOLVED, FALLBACK_CHECK_GOT, DECIDE, REJECT_GOT, FINISH, DONE
    };
    enum Need : uint8_t { NOTHING, ASSEMBLE, SOLVE };
    Stage stage = DONE;
    Need need = NOTHING;
    // device requests of the coming round
    bool mapping = true, consistent = false, x0zero = false, accept = false;
    uint32_t ops = 0;  // GATE_* copies and updates
    // newton()'s locals
    bool linearAllowed = true, converged = false, predictorUnloaded = false, handedOff = false, fellBack = true;
    double accepted = 0, opening = 0, lowest = 0;
    uint32_t loadingBefore = 0, solves = 0, attempt = 0, read = 0;
    tl_step_report rep{};
  };

  // Runs body `nb`'s control flow from its stage until it needs the device:
  // an assembly (need ASSEMBLE), a solve (need SOLVE) or nothing (DONE).
  // `squared`/`loadingNow` are the results of the assembly just made,
  // `moved`/`extent` those of the acceptance after the solve just made.
  void newtonAdvance(NewtonBody& nb, uint32_t cap, double travel, double squared, uint32_t loadingNow, double moved,
                     double extent) {
    using NB = NewtonBody;
    nb.need = NB::NOTHING;
    for (;;) {
      switch (nb.stage) {
        case NB::START:
          nb.ops |= GATE_ZERO_TOTAL;
          nb.accepted = std::numeric_limits<double>::infinity();
          nb.opening = 0.0;
          nb.lowest = std::numeric_limits<double>::infinity();
          nb.loadingBefore = 0;
          nb.solves = 0;
          nb.converged = nb.predictorUnloaded = nb.handedOff = false;
          nb.attempt = 0;
          nb.stage = NB::ATTEMPT;
          break;
        case NB::ATTEMPT:
          if (nb.attempt == cap) {
            nb.stage = NB::AFTER;
            break;
          }
          if (nb.attempt < 2u) nb.consistent = nb.attempt != 0u;
          nb.need = NB::ASSEMBLE;
          nb.mapping = true;
          nb.stage = NB::ATTEMPT_GOT;
          return;
        case NB::ATTEMPT_GOT: {
          ++nb.rep.plastic_evaluations;
          if (nb.attempt != 0u) {
            const double ranked = std::isfinite(squared) ? squared : std::numeric_limits<double>::infinity();
            if (nb.attempt == 1u || ranked < nb.lowest) {
              nb.lowest = ranked;
              nb.ops |= GATE_LOWEST_FROM_TOTAL;
            }
          }
          if (nb.attempt == 0u) nb.predictorUnloaded = loadingNow == 0u;
          if (nb.attempt == 1u && nb.linearAllowed && nb.predictorUnloaded && std::isfinite(squared) &&
              squared > nb.accepted) {
            ++nb.rep.plastic_linear_reads;
            nb.consistent = false;
            nb.read = 1;
            nb.stage = NB::LINEAR;
            break;
          }
          if (nb.attempt != 0u && !(squared <= nb.accepted)) {
            nb.ops |= GATE_BACKTRACK;
            ++nb.rep.plastic_backtracks;
            ++nb.attempt;
            nb.stage = NB::ATTEMPT;
            break;
          }
          if (nb.attempt != 0u && nb.loadingBefore == 0u && loadingNow == 0u) {
            nb.converged = true;
            nb.stage = NB::AFTER;
            break;
          }
          nb.opening = nb.attempt == 0u ? squared : nb.opening;
          nb.accepted = squared;
          nb.loadingBefore = loadingNow;
          if (nb.attempt == 0u) nb.ops |= GATE_INCR_FROM_A;
          nb.need = NB::SOLVE;
          nb.x0zero = nb.attempt != 0u;
          nb.accept = true;
          ++nb.solves;
          nb.stage = NB::ATTEMPT_SOLVED;
          return;
        }
        case NB::ATTEMPT_SOLVED:
          if (nb.solves > 1u &&
              travel * moved <= PLASTIC_RESOLUTION * double(std::numeric_limits<float>::epsilon()) * extent) {
            nb.converged = true;
            nb.stage = NB::AFTER;
            break;
          }
          ++nb.attempt;
          nb.stage = NB::ATTEMPT;
          break;
        case NB::LINEAR:
          if (nb.read == ANCHORED_READS) {
            nb.converged = !nb.handedOff;
            nb.stage = NB::AFTER;
            break;
          }
          nb.need = NB::ASSEMBLE;
          nb.mapping = true;
          nb.stage = NB::LINEAR_GOT;
          return;
        case NB::LINEAR_GOT:
          ++nb.rep.plastic_evaluations;
          if (loadingNow != 0u) {
            nb.handedOff = true;
            nb.converged = false;
            nb.stage = NB::AFTER;
            break;
          }
          nb.need = NB::SOLVE;
          nb.x0zero = true;
          nb.accept = false;
          ++nb.solves;
          nb.stage = NB::LINEAR_SOLVED;
          return;
        case NB::LINEAR_SOLVED:
          ++nb.read;
          nb.stage = NB::LINEAR;
          break;
        case NB::AFTER:
          nb.rep.plastic_solves += nb.solves;
          if (nb.handedOff) {
            ++nb.rep.plastic_handoffs;
            nb.linearAllowed = false;
            nb.stage = NB::START;
            break;
          }
          if (!nb.converged) {
            nb.consistent = false;
            nb.ops |= GATE_ZERO_TOTAL;
            nb.fellBack = true;
            nb.read = 0;
            nb.stage = NB::FALLBACK;
            break;
          }
          nb.stage = NB::FINISH;
          break;
        case NB::FALLBACK:
          nb.need = NB::ASSEMBLE;
          if (nb.read == ANCHORED_READS) {
            nb.mapping = true;
            nb.stage = NB::FALLBACK_CHECK_GOT;
          } else {
            nb.mapping = nb.read != 0u;
            nb.stage = NB::FALLBACK_GOT;
          }
          return;
        case NB::FALLBACK_GOT:
          ++nb.rep.plastic_evaluations;
          if (loadingNow != 0u) {
            nb.fellBack = false;
            nb.stage = NB::DECIDE;
            break;
          }
          if (nb.read == 0u) nb.ops |= GATE_INCR_FROM_A;
          nb.need = NB::SOLVE;
          nb.x0zero = nb.read != 0u;
          nb.accept = false;
          ++nb.rep.plastic_solves;
          nb.stage = NB::FALLBACK_SOLVED;
          return;
        case NB::FALLBACK_SOLVED:
          ++nb.read;
          nb.stage = NB::FALLBACK;
          break;
        case NB::FALLBACK_CHECK_GOT:
          ++nb.rep.plastic_evaluations;
          nb.fellBack = loadingNow == 0u && squared <= PLASTIC_REDUCTION * PLASTIC_REDUCTION * nb.opening;
          nb.stage = NB::DECIDE;
          break;
        case NB::DECIDE:
          if (nb.fellBack) {
            ++nb.rep.plastic_fallbacks;
            nb.converged = true;
            nb.stage = NB::FINISH;
            break;
          }
          ++nb.rep.plastic_fallback_rejections;
          nb.consistent = true;
          nb.ops |= GATE_TOTAL_FROM_LOWEST;
          nb.need = NB::ASSEMBLE;
          nb.mapping = true;
          nb.stage = NB::REJECT_GOT;
          return;
        case NB::REJECT_GOT: {
          ++nb.rep.plastic_evaluations;
          const double remaining = std::sqrt(nb.lowest);
          if (remaining >= nb.rep.plastic_worst_residual) nb.rep.plastic_worst_residual = remaining;
          nb.stage = NB::FINISH;
          break;
        }
        case NB::FINISH:
          nb.rep.plastic_capped += nb.converged ? 0u : 1u;
          nb.ops |= GATE_A_FROM_TOTAL;
          nb.stage = NB::DONE;
          return;
        case NB::DONE:
          return;
      }
    }
  }

  // Launches `k` for the bodies whose pending ops carry `bit` (once per round).
  void gatedNodeCopy(uint32_t bit, DevBuf<Vec4<S>>& dst, const Vec4<S>* src, uint32_t pass) {
    gateBit = bit;
    kNodeCopy<S><<<nodeTiles, TILE, 0, st>>>(view(), dst.ptr, src, pass);
    gateBit = 0;
    check();
  }
  void uploadGates() {
    gate.upload(hGate.ptr, B, st);
  }

  std::vector<NewtonBody> nbs;
  std::vector<uint32_t> newtonYielding;  // each Newton body's yielding count at its last assembly

  void newtonBatch(int law, uint32_t pass, const tl_settings& set, const Rule& rule, const BodyStepDev* hs,
                   std::vector<tl_step_report>& local, const std::vector<uint8_t>& newtonBody) {
    using NB = NewtonBody;
    if (!gate.ptr) gate.alloc(B);
    uint32_t* hg = hGate.get(B);
    nbs.assign(B, NB{});
    newtonYielding.assign(B, 0u);
    bool anyElastic = false;
    for (uint32_t b = 0; b < B; ++b) {
      if (pass >= hs[b].substeps) continue;
      if (!newtonBody[b]) {
        anyElastic = true;
        continue;
      }
      nbs[b].stage = NB::START;
      newtonAdvance(nbs[b], set.plastic_passes, rule.beta * hs[b].inner * hs[b].inner, 0, 0, 0, 0);
    }
    // the batch's elastic bodies take the three reads on their own gate
    if (anyElastic) {
      for (uint32_t b = 0; b < B; ++b) hg[b] = (pass < hs[b].substeps && !newtonBody[b]) ? GATE_ELASTIC : 0u;
      uploadGates();
      gateBit = GATE_ELASTIC;
      try {
        elasticReads(law, pass);
      } catch (...) {
        gateBit = 0;
        throw;
      }
      gateBit = 0;
    }
    for (;;) {
      // ---- pre-assembly updates and the assembly
      uint32_t orAll = 0;
      bool anyAssemble = false;
      for (uint32_t b = 0; b < B; ++b) {
        NB& nb = nbs[b];
        uint32_t w = nb.ops & (GATE_ZERO_TOTAL | GATE_TOTAL_FROM_LOWEST | GATE_BACKTRACK | GATE_A_FROM_TOTAL);
        nb.ops &= ~w;
        if (nb.need == NB::ASSEMBLE) {
          w |= GATE_ASSEMBLE | (nb.mapping ? uint32_t(EM_MAPPING) : 0u) | (nb.consistent ? uint32_t(EM_CONSISTENT) : 0u);
          anyAssemble = true;
        }
        hg[b] = w;
        orAll |= w;
      }
      if (orAll) uploadGates();
      if (orAll & GATE_ZERO_TOTAL) gatedNodeCopy(GATE_ZERO_TOTAL, total, nullptr, pass);
      if (orAll & GATE_TOTAL_FROM_LOWEST) gatedNodeCopy(GATE_TOTAL_FROM_LOWEST, total, lowest.ptr, pass);
      if (orAll & GATE_BACKTRACK) {
        gateBit = GATE_BACKTRACK;
        nodeOp(kBacktrack<S>, pass);
        gateBit = 0;
      }
      if (orAll & GATE_A_FROM_TOTAL) gatedNodeCopy(GATE_A_FROM_TOTAL, a, total.ptr, pass);
      if (anyAssemble) {
        gateBit = GATE_ASSEMBLE;
        try {
          element(law, weighted.ptr, total.ptr, pass, EM_MAPPING, LOADING_MARGIN);
          nodeAssemble(total.ptr, pass);
        } catch (...) {
          gateBit = 0;
          throw;
        }
        gateBit = 0;
        finalize(1);
        BodyAccDev* ha = hAcc.get(B);
        uint32_t* hc = hCount.get(2 * size_t(B));
        acc.download(ha, B, st);
        loading.download(hc, B, st);
        yielding.download(hc + B, B, st);
        TL_CUDA(cudaStreamSynchronize(st));
        for (uint32_t b = 0; b < B; ++b) {
          NB& nb = nbs[b];
          if (nb.need != NB::ASSEMBLE) continue;
          newtonYielding[b] = hc[B + b];
          newtonAdvance(nb, set.plastic_passes, rule.beta * hs[b].inner * hs[b].inner, ha[b].right_sq, hc[b], 0, 0);
        }
      }
      // ---- copies before the solves, the solves by launch group, the updates after them
      orAll = 0;
      bool anySolve = false, anyAccept = false;
      uint32_t groups = 0;
      for (uint32_t b = 0; b < B; ++b) {
        NB& nb = nbs[b];
        uint32_t w = nb.ops & (GATE_LOWEST_FROM_TOTAL | GATE_INCR_FROM_A | GATE_A_FROM_TOTAL);
        nb.ops &= ~w;
        if (nb.need == NB::SOLVE) {
          const uint32_t g = (nb.x0zero ? 1u : 0u) + (nb.consistent ? 2u : 0u);
          w |= (GATE_SOLVE0 << g) | (nb.accept ? GATE_ACCEPT : GATE_ADD);
          groups |= 1u << g;
          anySolve = true;
          anyAccept = anyAccept || nb.accept;
        }
        hg[b] = w;
        orAll |= w;
      }
      if (orAll) uploadGates();
      if (orAll & GATE_LOWEST_FROM_TOTAL) gatedNodeCopy(GATE_LOWEST_FROM_TOTAL, lowest, total.ptr, pass);
      if (orAll & GATE_INCR_FROM_A) gatedNodeCopy(GATE_INCR_FROM_A, incr, a.ptr, pass);
      if (orAll & GATE_A_FROM_TOTAL) gatedNodeCopy(GATE_A_FROM_TOTAL, a, total.ptr, pass);
      if (anySolve) {
        for (uint32_t g = 0; g < 4u; ++g) {
          if (!(groups & (1u << g))) continue;
          gateBit = GATE_SOLVE0 << g;
          try {
            pcg(law, incr.ptr, pass, (g & 1u) != 0u, (g & 2u) != 0u);
          } catch (...) {
            gateBit = 0;
            throw;
          }
          gateBit = 0;
        }
        if (anyAccept) {
          kAccMovedReset<<<(B + 255) / 256, 256, 0, st>>>(acc.ptr, B);
          check();
          gateBit = GATE_ACCEPT;
          nodeOp(kNewtonAccept<S>, pass);
          gateBit = 0;
        }
        if (orAll & GATE_ADD) {
          gateBit = GATE_ADD;
          kAddIncrement<S><<<nodeTiles, TILE, 0, st>>>(view(), total.ptr, pass);
          gateBit = 0;
          check();
        }
        BodyAccDev* ha = hAcc.get(B);
        acc.download(ha, B, st);
        TL_CUDA(cudaStreamSynchronize(st));
        for (uint32_t b = 0; b < B; ++b) {
          NB& nb = nbs[b];
          if (nb.need != NB::SOLVE) continue;
          double moved = 0.0, extent = 0.0;
          if (nb.accept) {
            std::memcpy(&moved, &ha[b].moved_key, 8);
            std::memcpy(&extent, &ha[b].extent_key, 8);
          }
          newtonAdvance(nb, set.plastic_passes, rule.beta * hs[b].inner * hs[b].inner, 0, 0, moved, extent);
        }
      }
      bool pending = false;
      for (const NB& nb : nbs) pending = pending || nb.need != NB::NOTHING || nb.ops != 0u;
      if (!pending) break;
    }
    for (uint32_t b = 0; b < B; ++b) {
      if (!newtonBody[b] || pass >= hs[b].substeps) continue;
      const tl_step_report& r = nbs[b].rep;
      tl_step_report& l = local[b];
      l.plastic_evaluations += r.plastic_evaluations;
      l.plastic_solves += r.plastic_solves;
      l.plastic_backtracks += r.plastic_backtracks;
      l.plastic_capped += r.plastic_capped;
      l.plastic_linear_reads += r.plastic_linear_reads;
      l.plastic_handoffs += r.plastic_handoffs;
      l.plastic_fallbacks += r.plastic_fallbacks;
      l.plastic_fallback_rejections += r.plastic_fallback_rejections;
      l.plastic_worst_residual = std::max(l.plastic_worst_residual, r.plastic_worst_residual);
      l.yielding = newtonYielding[b];
    }
  }

  // Per-element E override (tl_system_set_youngs).  The first call gives
  // every element its lane's modulus, then overwrites the body's elements.
  void setYoungs(uint32_t b, const double* E) override {
    const BodyDev& bd = bodyHost[b];
    const HostBody& h = hb[b];
    for (uint32_t t = 0; t < h.tets; ++t)
      if (!(E[t] > 0.0) || !std::isfinite(E[t])) throw StatusError{TL_ERR_ARG, "Young's modulus must be positive"};
    if (!hasEyoung) {
      eyoung.alloc(Tp);
      kLaneYoungs<<<elemTiles, TILE, 0, st>>>(view(), eyoung.ptr);
      TL_CUDA(cudaGetLastError());
      hasEyoung = true;
      if (graphExec) cudaGraphExecDestroy(graphExec);  // the captured launches hold the old element view
      graphExec = nullptr;
    }
    eyoung.upload(E, h.tets, st, bd.elem_begin);
    if (b == 0) fYoungs.assign(E, E + h.tets);
    TL_CUDA(cudaStreamSynchronize(st));
  }

  std::unique_ptr<RolloutBase> rollout(const tl_rollout_desc& desc, const tl_settings& settings) override;

  // tl_evaluate: one element pass at the resident positions and the force
  // gather, with the committed rotations put back afterwards.
  uint8_t* yflagPtr = nullptr;
  void evaluate(uint32_t b, const tl_settings& set, double* forces, uint8_t* yielding) override {
    if (set.law > 1u) throw StatusError{TL_ERR_ARG, "unknown law"};
    if (hencky && set.law != TL_LAW_COROTATED)
      throw StatusError{TL_ERR_UNSUPPORTED, "the plastic rest shape is written for the corotated law"};
    const BodyDev& bd = bodyHost[b];
    const HostBody& h = hb[b];
    BodyStepDev* hs = hStep.get(B);
    for (uint32_t k = 0; k < B; ++k) {
      std::memset(&hs[k], 0, sizeof(BodyStepDev));
      hs[k].substeps = 1;
    }
    dStep.upload(hs, B, st);
    DevBuf<S> keepOp;
    keepOp.alloc(size_t(9) * Tp);
    TL_CUDA(cudaMemcpyAsync(keepOp.ptr, op.ptr, sizeof(S) * 9 * size_t(Tp), cudaMemcpyDeviceToDevice, st));
    DevBuf<uint8_t> flags;
    DevBuf<double> out;
    flags.alloc(Tp);
    out.alloc(size_t(3) * Vp);
    yflagPtr = flags.ptr;
    try {
      evaluating = true;
      element(int(set.law), u.ptr, nullptr, 0, EM_MAPPING, 0.0);
      evaluating = false;
    } catch (...) {
      yflagPtr = nullptr;
      evaluating = false;
      throw;
    }
    yflagPtr = nullptr;
    kGatherForces<S><<<nodeTiles, TILE, 0, st>>>(view(), out.ptr);
    check();
    TL_CUDA(cudaMemcpyAsync(op.ptr, keepOp.ptr, sizeof(S) * 9 * size_t(Tp), cudaMemcpyDeviceToDevice, st));
    if (forces) out.download(forces, size_t(3) * h.nodes, st, size_t(3) * bd.node_begin);
    if (yielding) flags.download(yielding, h.tets, st, bd.elem_begin);
    TL_CUDA(cudaStreamSynchronize(st));
  }
};

// Checkpointed rollout and its adjoint (kernels and equations in
// tl_adjoint.cuh).  State layout of a stored state: u, v, a, each [Vp].
template <class S>
struct Rollout final : RolloutBase {
  System<S>& sys;
  tl_rollout_desc d;
  tl_settings set;
  uint32_t segments = 0;
  size_t stride = 0;  // elements of one stored state
  DevBuf<Vec4<S>> ck, seg, fin, xb, vb, ab, lam;
  DevBuf<double> ebar;
  bool ran = false;

  Rollout(System<S>& s, const tl_rollout_desc& desc, const tl_settings& settings) : sys(s), d(desc), set(settings) {
    if (sys.B != 1u) throw StatusError{TL_ERR_UNSUPPORTED, "a rollout runs on a one-body system"};
    if (sys.hencky) throw StatusError{TL_ERR_UNSUPPORTED, "a rollout does not differentiate the plastic flow"};
    if (settings.law != TL_LAW_SNH)
      throw StatusError{TL_ERR_UNSUPPORTED, "the adjoint needs the exact tangent of TL_LAW_SNH"};
    if (sys.hb[0].floats(settings.rigid_split))
      throw StatusError{TL_ERR_UNSUPPORTED, "the adjoint does not differentiate the floating frame"};
    if (!desc.steps || !desc.checkpoint_every || !desc.newton_reads || !(desc.delta_time > 0.0))
      throw StatusError{TL_ERR_ARG, "rollout needs steps, checkpoint_every, newton_reads >= 1 and dt > 0"};
    segments = (desc.steps + desc.checkpoint_every - 1) / desc.checkpoint_every;
    stride = size_t(3) * sys.Vp;
    ck.alloc(stride * segments);
    seg.alloc(stride * (size_t(std::min(desc.checkpoint_every, desc.steps)) + 1));
    fin.alloc(stride);
    for (DevBuf<Vec4<S>>* b : {&xb, &vb, &ab, &lam}) {
      b->alloc(sys.Vp);
      b->zero(sys.st);
    }
    ebar.alloc(sys.Tp);
  }

  void save(Vec4<S>* dst) {
    const size_t bytes = size_t(sys.Vp) * sizeof(Vec4<S>);
    TL_CUDA(cudaMemcpyAsync(dst, sys.u.ptr, bytes, cudaMemcpyDeviceToDevice, sys.st));
    TL_CUDA(cudaMemcpyAsync(dst + sys.Vp, sys.v.ptr, bytes, cudaMemcpyDeviceToDevice, sys.st));
    TL_CUDA(cudaMemcpyAsync(dst + 2 * size_t(sys.Vp), sys.a.ptr, bytes, cudaMemcpyDeviceToDevice, sys.st));
  }
  void load(const Vec4<S>* src) {
    const size_t bytes = size_t(sys.Vp) * sizeof(Vec4<S>);
    TL_CUDA(cudaMemcpyAsync(sys.u.ptr, src, bytes, cudaMemcpyDeviceToDevice, sys.st));
    TL_CUDA(cudaMemcpyAsync(sys.v.ptr, src + sys.Vp, bytes, cudaMemcpyDeviceToDevice, sys.st));
    TL_CUDA(cudaMemcpyAsync(sys.a.ptr, src + 2 * size_t(sys.Vp), bytes, cudaMemcpyDeviceToDevice, sys.st));
  }

  void stepOnce(tl_step_report* report) {
    tl_step_report local;
    std::memset(&local, 0, sizeof(local));
    tl_step_report* r = report ? report : &local;
    const uint64_t before = r->substeps;
    sys.newtonReads = d.newton_reads;
    int32_t rc;
    try {
      rc = sys.step(set, d.gravity, d.delta_time, r);
    } catch (...) {
      sys.newtonReads = ANCHORED_READS;
      throw;
    }
    sys.newtonReads = ANCHORED_READS;
    if (rc == TL_ERR_NONFINITE) throw StatusError{TL_ERR_NONFINITE, "the rollout state became non-finite"};
    if (rc != TL_OK) throw StatusError{rc, "rollout step failed"};
    if (r->substeps - before != 1u)
      throw StatusError{TL_ERR_UNSUPPORTED, "a rollout step needed more than one substep (predictor inversion)"};
  }

  void forward(tl_step_report* report, double* seconds) override {
    cudaEvent_t e0, e1;
    TL_CUDA(cudaEventCreate(&e0));
    TL_CUDA(cudaEventCreate(&e1));
    TL_CUDA(cudaEventRecord(e0, sys.st));
    save(ck.ptr);
    const uint32_t C = d.checkpoint_every;
    for (uint32_t n = 0; n < d.steps; ++n) {
      stepOnce(report);
      if ((n + 1) % C == 0 && n + 1 < d.steps) save(ck.ptr + stride * ((n + 1) / C));
    }
    save(fin.ptr);
    TL_CUDA(cudaEventRecord(e1, sys.st));
    TL_CUDA(cudaStreamSynchronize(sys.st));
    float ms = 0.f;
    TL_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (seconds) *seconds = double(ms) * 1e-3;
    ran = true;
  }

  void adjoint(const double* dxT, const double* dvT, double* dE, double* dv0, double* dx0,
               double* seconds) override {
    if (!ran) throw StatusError{TL_ERR_ARG, "tl_rollout_adjoint needs a forward rollout first"};
    const BodyDev& bd = sys.bodyHost[0];
    const HostBody& h = sys.hb[0];
    xb.zero(sys.st);
    vb.zero(sys.st);
    ab.zero(sys.st);
    ebar.zero(sys.st);
    TL_CUDA(cudaMemsetAsync(&sys.sync.ptr->error, 0, sizeof(int), sys.st));
    if (dxT) sys.setNodes(bd, h, xb, dxT, false);
    if (dvT) sys.setNodes(bd, h, vb, dvT, false);
    cudaEvent_t e0, e1;
    TL_CUDA(cudaEventCreate(&e0));
    TL_CUDA(cudaEventCreate(&e1));
    TL_CUDA(cudaEventRecord(e0, sys.st));
    const uint32_t C = d.checkpoint_every;
    for (uint32_t k = segments; k-- > 0;) {
      const uint32_t s0 = k * C, s1 = std::min(d.steps, s0 + C), L = s1 - s0;
      // recompute the segment from its checkpoint, keeping every state
      load(ck.ptr + stride * k);
      save(seg.ptr);
      for (uint32_t j = 0; j < L; ++j) {
        stepOnce(nullptr);
        save(seg.ptr + stride * (j + 1));
      }
      for (uint32_t j = L; j-- > 0;) {
        load(seg.ptr + stride * j);
        const Vec4<S>* A = seg.ptr + stride * (j + 1) + 2 * size_t(sys.Vp);  // converged acceleration of step j
        sys.nodeOp(kPredict<S>, 0);
        sys.element(TL_LAW_SNH, sys.weighted.ptr, A, 0, EM_MAPPING, 0.0);
        sys.nodeAssemble(A, 0);
        kAdjointRight<S><<<sys.nodeTiles, TILE, 0, sys.st>>>(sys.view(), xb.ptr, vb.ptr, ab.ptr);
        sys.check();
        sys.pcg(TL_LAW_SNH, lam.ptr, 0, true, false);
        kAdjointElement<S, 1><<<sys.elemTiles, TILE, 0, sys.st>>>(sys.view(), lam.ptr, ebar.ptr);
        sys.check();
        kAdjointNode<S><<<sys.nodeTiles, TILE, 0, sys.st>>>(sys.view(), lam.ptr, xb.ptr, vb.ptr, ab.ptr);
        sys.check();
      }
      GridSyncDev* hs = sys.hSync.get(1);
      sys.sync.download(hs, 1, sys.st);
      TL_CUDA(cudaStreamSynchronize(sys.st));
      if (hs->error != 0) throw StatusError{TL_ERR_TIMEOUT, "a PCG grid barrier ran out of time"};
    }
    load(fin.ptr);
    TL_CUDA(cudaEventRecord(e1, sys.st));
    TL_CUDA(cudaStreamSynchronize(sys.st));
    float ms = 0.f;
    TL_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (seconds) *seconds = double(ms) * 1e-3;
    if (dE) {
      ebar.download(dE, h.tets, sys.st, bd.elem_begin);
      TL_CUDA(cudaStreamSynchronize(sys.st));
    }
    if (dv0) sys.getNodes(bd, h, vb, dv0, false);
    if (dx0) sys.getNodes(bd, h, xb, dx0, false);
  }
};

template <class S>
std::unique_ptr<RolloutBase> System<S>::rollout(const tl_rollout_desc& desc, const tl_settings& settings) {
  return std::make_unique<Rollout<S>>(*this, desc, settings);
}

int32_t fail(tl_ctx* ctx, int32_t status, const std::string& what) {
  if (ctx) ctx->last_error = what;
  return status;
}

template <class F>
int32_t guarded(tl_ctx* ctx, F&& body) {
  try {
    return body();
  } catch (const StatusError& e) {
    return fail(ctx, e.status, e.what);
  } catch (const CudaError& e) {
    return fail(ctx, TL_ERR_CUDA, std::string(e.what) + ": " + cudaGetErrorString(e.code));
  } catch (const std::bad_alloc&) {
    return fail(ctx, TL_ERR_ARG, "host allocation failed");
  }
}

}  // namespace

extern "C" {

int32_t tl_abi_version(void) { return TL_ABI_VERSION; }

const char* tl_status_string(int32_t status) {
  switch (status) {
    case TL_OK: return "ok";
    case TL_ERR_ARG: return "invalid argument";
    case TL_ERR_CUDA: return "CUDA error";
    case TL_ERR_NOT_CONVERGED: return "not converged";
    case TL_ERR_NONFINITE: return "non-finite state";
    case TL_ERR_TIMEOUT: return "device wait timed out";
    case TL_ERR_UNSUPPORTED: return "unsupported";
    case TL_ERR_NO_DEVICE: return "no CUDA device";
    case TL_ERR_TOO_LARGE: return "input exceeds the fixed capacity of tl_step_noalloc";
    default: return "unknown status";
  }
}

void tl_settings_default(tl_settings* s) {
  if (!s) return;
  s->substeps = 1u;
  s->cg_iterations = 64u;
  s->plastic_passes = 40u;
  s->rigid_split = TL_RIGID_SPLIT_PROJECTED;
  s->law = TL_LAW_COROTATED;
  s->flags = 0u;
  s->tolerance = 1.0e-3;
  s->spectral_radius = 0.5;
}

int32_t tl_ctx_create(int32_t device, tl_ctx** out) {
  if (!out) return TL_ERR_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) return TL_ERR_NO_DEVICE;
  if (device < 0 || device >= count) return TL_ERR_ARG;
  auto ctx = std::make_unique<tl_ctx>();
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess) return TL_ERR_NO_DEVICE;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return TL_ERR_NO_DEVICE;
  if (prop.major < 10) return TL_ERR_NO_DEVICE;  // built for sm_100a only
  int coop = 0;
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
  if (!coop) return TL_ERR_NO_DEVICE;
  ctx->sms = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) return TL_ERR_CUDA;
  *out = ctx.release();
  return TL_OK;
}

int32_t tl_ctx_destroy(tl_ctx* ctx) {
  if (!ctx) return TL_ERR_ARG;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return TL_OK;
}

const char* tl_ctx_last_error(const tl_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

}  // extern "C"

extern "C" {

int32_t tl_ctx_check_wait_limit(tl_ctx* ctx) {
  if (!ctx) return TL_ERR_ARG;
  return guarded(ctx, [&]() -> int32_t {
    TL_CUDA(cudaSetDevice(ctx->device));
    DevBuf<GridSyncDev> sync;
    sync.alloc(1);
    sync.zero(ctx->stream);
    kWaitLimitCheck<<<1, TILE, 0, ctx->stream>>>(sync.ptr);
    TL_CUDA(cudaGetLastError());
    GridSyncDev h{};
    sync.download(&h, 1, ctx->stream);
    TL_CUDA(cudaStreamSynchronize(ctx->stream));
    if (h.error != 0) return fail(ctx, TL_ERR_TIMEOUT, "the grid barrier's bounded wait ran out (self test)");
    return TL_OK;
  });
}

int32_t tl_system_create(tl_ctx* ctx, const tl_mesh_desc* bodies, uint32_t count, int32_t precision,
                         tl_system** out) {
  if (!ctx || !bodies || !count || !out) return TL_ERR_ARG;
  *out = nullptr;
  return guarded(ctx, [&]() -> int32_t {
    TL_CUDA(cudaSetDevice(ctx->device));
    auto sys = std::make_unique<tl_system>();
    sys->ctx = ctx;
    sys->device = ctx->device;
    if (precision == TL_FP64) sys->impl = std::make_unique<System<double>>(ctx, bodies, count);
    else if (precision == TL_FP32_MIXED) sys->impl = std::make_unique<System<float>>(ctx, bodies, count);
    else return fail(ctx, TL_ERR_ARG, "unknown precision");
    *out = sys.release();
    return TL_OK;
  });
}

int32_t tl_system_destroy(tl_system* system) {
  if (!system) return TL_ERR_ARG;
  cudaSetDevice(system->device);
  cudaDeviceSynchronize();
  delete system;
  return TL_OK;
}

int32_t tl_system_counts(const tl_system* system, uint32_t* bodies, uint64_t* nodes, uint64_t* tets) {
  if (!system) return TL_ERR_ARG;
  if (bodies) *bodies = system->impl->bodies;
  if (nodes) *nodes = system->impl->nodes;
  if (tets) *tets = system->impl->tets;
  return TL_OK;
}

int32_t tl_system_tune(tl_system* system, uint32_t pcg_blocks_per_sm, uint32_t graph) {
  if (!system || pcg_blocks_per_sm > 64u) return TL_ERR_ARG;
  return guarded(system->ctx, [&]() -> int32_t {
    TL_CUDA(cudaSetDevice(system->ctx->device));
    system->impl->tune(pcg_blocks_per_sm, graph);
    return TL_OK;
  });
}

int32_t tl_system_tune_shape(tl_system* system, uint32_t knob, uint32_t value) {
  if (!system) return TL_ERR_ARG;
  return guarded(system->ctx, [&]() -> int32_t {
    TL_CUDA(cudaSetDevice(system->ctx->device));
    system->impl->tuneShape(knob, value);
    return TL_OK;
  });
}

int32_t tl_system_expire_wait(tl_system* system, int32_t solve) {
  if (!system) return TL_ERR_ARG;
  system->impl->expireWait(solve < 0 ? -1 : solve);
  return TL_OK;
}

int32_t tl_system_set_solver(tl_system* system, uint32_t form) {
  if (!system || form > TL_SOLVER_ASSEMBLED_PIPELINED) return TL_ERR_ARG;
  return guarded(system->ctx, [&]() -> int32_t {
    system->impl->setSolver(form);
    return TL_OK;
  });
}

int32_t tl_system_use_factor(tl_system* system, uint32_t enable, uint32_t factor_budget) {
  if (!system) return TL_ERR_ARG;
  return guarded(system->ctx, [&]() -> int32_t {
    TL_CUDA(cudaSetDevice(system->ctx->device));
    system->impl->useFactor(enable, factor_budget);
    return TL_OK;
  });
}

int32_t tl_system_factor_stats(tl_system* system, tl_factor_stats* out) {
  if (!system || !out) return TL_ERR_ARG;
  return guarded(system->ctx, [&]() -> int32_t {
    system->impl->factorStats(out);
    return TL_OK;
  });
}

int32_t tl_system_set_plasticity(tl_system* system, uint32_t mode) {
  if (!system || mode > TL_PLASTICITY_HENCKY) return TL_ERR_ARG;
  return guarded(system->ctx, [&]() -> int32_t {
    TL_CUDA(cudaSetDevice(system->ctx->device));
    system->impl->setPlasticity(mode);
    return TL_OK;
  });
}

int32_t tl_system_set_flow_limits(tl_system* system, uint32_t body, uint32_t lane, double crush_stress,
                                  double crush_limit, double plastic_max) {
  // crushStress > 0 (+inf: none), crushLimit in (0, 1] (1: none), plasticMax > 0 (+inf: none)
  if (!system || std::isnan(crush_stress) || !(crush_stress > 0.0) || !(crush_limit > 0.0) ||
      !(crush_limit <= 1.0) || std::isnan(plastic_max) || !(plastic_max > 0.0))
    return TL_ERR_ARG;
  return guarded(system->ctx, [&]() -> int32_t {
    TL_CUDA(cudaSetDevice(system->ctx->device));
    system->impl->setFlowLimits(body, lane, crush_stress, crush_limit, plastic_max);
    return TL_OK;
  });
}

int32_t tl_step_substeps(const tl_system* system, uint32_t body, uint32_t* iterations, double* start_residual,
                         double* end_residual, uint32_t capacity, uint32_t* count) {
  if (!system || body >= system->impl->bodies) return TL_ERR_ARG;
  const SystemBase& s = *system->impl;
  const uint32_t taken = s.substepCounts.empty() ? 0u : s.substepCounts[body];
  const uint32_t kept = std::min({capacity, taken, SUBSTEP_RECORDS});
  for (uint32_t k = 0; k < kept; ++k) {
    const SubstepRecordDev& r = s.substepRecords[size_t(body) * SUBSTEP_RECORDS + k];
    if (iterations) iterations[k] = r.iterations;
    if (start_residual) start_residual[k] = r.start_residual;
    if (end_residual) end_residual[k] = r.end_residual;
  }
  if (count) *count = taken;
  return TL_OK;
}

int32_t tl_system_trace(const tl_system* system, uint32_t* iterations, uint32_t capacity, uint32_t* count) {
  if (!system || (capacity && !iterations)) return TL_ERR_ARG;
  const std::vector<uint32_t>& t = system->impl->trace;
  const size_t n = std::min<size_t>(capacity, t.size());
  std::copy(t.begin(), t.begin() + n, iterations);
  if (count) *count = uint32_t(t.size());
  return TL_OK;
}

int32_t tl_state_set(tl_system* system, uint32_t body, int32_t dtype, const void* position, const void* velocity,
                     const void* acceleration, const void* rotation, const void* plastic) {
  if (!system || body >= system->impl->bodies || (dtype != TL_DTYPE_F32 && dtype != TL_DTYPE_F64)) return TL_ERR_ARG;
  return guarded(system->ctx, [&]() -> int32_t {
    TL_CUDA(cudaSetDevice(system->ctx->device));
    system->impl->stateSet(body, dtype, position, velocity, acceleration, rotation, plastic);
    return TL_OK;
  });
}

int32_t tl_state_get(tl_system* system, uint32_t body, int32_t dtype, void* position, void* velocity,
                     void* acceleration, void* rotation, void* plastic) {
  if (!system || body >= system->impl->bodies || (dtype != TL_DTYPE_F32 && dtype != TL_DTYPE_F64)) return TL_ERR_ARG;
  return guarded(system->ctx, [&]() -> int32_t {
    TL_CUDA(cudaSetDevice(system->ctx->device));
    system->impl->stateGet(body, dtype, position, velocity, acceleration, rotation, plastic);
    return TL_OK;
  });
}

int32_t tl_step(tl_system* system, const tl_settings* settings, const double gravity[3], double dt,
                tl_step_report* reports) {
  if (!system || !settings || !gravity || !stepArgumentsValid(dt, gravity)) return TL_ERR_ARG;
  return guarded(system->ctx, [&]() -> int32_t {
    TL_CUDA(cudaSetDevice(system->ctx->device));
    return system->impl->step(*settings, gravity, dt, reports);
  });
}

int32_t tl_evaluate(tl_system* system, uint32_t body, const tl_settings* settings, double* forces,
                    uint8_t* yielding) {
  if (!system || !settings || body >= system->impl->bodies) return TL_ERR_ARG;
  return guarded(system->ctx, [&]() -> int32_t {
    TL_CUDA(cudaSetDevice(system->ctx->device));
    system->impl->evaluate(body, *settings, forces, yielding);
    return TL_OK;
  });
}

int32_t tl_system_set_youngs(tl_system* system, uint32_t body, const double* youngs) {
  if (!system || !youngs || body >= system->impl->bodies) return TL_ERR_ARG;
  return guarded(system->ctx, [&]() -> int32_t {
    TL_CUDA(cudaSetDevice(system->ctx->device));
    system->impl->setYoungs(body, youngs);
    return TL_OK;
  });
}

int32_t tl_rollout_create(tl_system* system, const tl_rollout_desc* desc, const tl_settings* settings,
                          tl_rollout** out) {
  if (!system || !desc || !settings || !out) return TL_ERR_ARG;
  *out = nullptr;
  return guarded(system->ctx, [&]() -> int32_t {
    TL_CUDA(cudaSetDevice(system->ctx->device));
    auto r = std::make_unique<tl_rollout>();
    r->system = system;
    r->device = system->device;
    r->impl = system->impl->rollout(*desc, *settings);
    *out = r.release();
    return TL_OK;
  });
}

int32_t tl_rollout_destroy(tl_rollout* rollout) {
  if (!rollout) return TL_ERR_ARG;
  cudaSetDevice(rollout->device);
  cudaDeviceSynchronize();
  delete rollout;
  return TL_OK;
}

int32_t tl_rollout_forward(tl_rollout* rollout, tl_step_report* report, double* device_seconds) {
  if (!rollout) return TL_ERR_ARG;
  return guarded(rollout->system->ctx, [&]() -> int32_t {
    TL_CUDA(cudaSetDevice(rollout->system->ctx->device));
    rollout->impl->forward(report, device_seconds);
    return TL_OK;
  });
}

int32_t tl_rollout_adjoint(tl_rollout* rollout, const double* dl_dx_final, const double* dl_dv_final,
                           double* dl_dyoungs, double* dl_dv0, double* dl_dx0, double* device_seconds) {
  if (!rollout) return TL_ERR_ARG;
  return guarded(rollout->system->ctx, [&]() -> int32_t {
    TL_CUDA(cudaSetDevice(rollout->system->ctx->device));
    rollout->impl->adjoint(dl_dx_final, dl_dv_final, dl_dyoungs, dl_dv0, dl_dx0, device_seconds);
    return TL_OK;
  });
}

int32_t tl_host_register(tl_ctx* ctx, void* ptr, size_t bytes) {
  if (!ctx || !ptr || !bytes) return TL_ERR_ARG;
  return guarded(ctx, [&]() -> int32_t {
    TL_CUDA(cudaSetDevice(ctx->device));
    TL_CUDA(cudaHostRegister(ptr, bytes, cudaHostRegisterDefault));
    return TL_OK;
  });
}

int32_t tl_host_unregister(tl_ctx* ctx, void* ptr) {
  if (!ctx || !ptr) return TL_ERR_ARG;
  return guarded(ctx, [&]() -> int32_t {
    TL_CUDA(cudaSetDevice(ctx->device));
    TL_CUDA(cudaHostUnregister(ptr));
    return TL_OK;
  });
}

int32_t tl_step_host(tl_system* system, uint32_t body, int32_t dtype, void* position, void* velocity,
                     void* acceleration, void* rotation, void* plastic, const tl_settings* settings,
                     const double gravity[3], double dt, tl_step_report* report) {
  if (!system || !settings || body >= system->impl->bodies || system->impl->bodies != 1u) return TL_ERR_ARG;
  // The incoming rotations are not uploaded: every element pass writes each
  // committed rotation before any kernel reads one (kElement, then kDamping
  // and the matvec), as assembleElastic does in the reference
  // (solver.cc:1404, 1446, 1500, 1547 before 745-987).  They are outputs only.
  // The plastic slot crosses only when the step reads it: with no yielding
  // lane under the corotated law (the SNH law runs elastic here) and the
  // small-strain mode, the step leaves the plastic points as they are, so the
  // caller's buffer already holds them.  In the finite-strain mode every tet's
  // plastic map shapes its rest, so the slot always crosses.
  const bool plasticUsed = system->impl->plasticUsed(settings->law);
  void* pl = plasticUsed ? plastic : nullptr;
  int32_t rc = tl_state_set(system, body, dtype, position, velocity, acceleration, nullptr, pl);
  if (rc != TL_OK) return rc;
  rc = tl_step(system, settings, gravity, dt, report);
  if (rc != TL_OK && rc != TL_ERR_NONFINITE) return rc;
  const int32_t got = tl_state_get(system, body, dtype, position, velocity, acceleration, rotation, pl);
  return got != TL_OK ? got : rc;
}

}  // extern "C"
