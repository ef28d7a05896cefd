// tl_kernels.cuh -- sm_100a kernels of the tet FEM step.
//
// Layout in HBM (one resident "system" = one or more bodies, concatenated):
//  * nodes: Vec4 records (x, y, z, w) so that one 16-byte (FP32) or 32-byte
//    (FP64) load moves a node vector; the state is stored as DISPLACEMENT
//    u = x - X from the rest position X, which keeps FP32 storage accurate
//    for small motions of large bodies.  Each body's nodes are padded to a
//    multiple of TILE; padding nodes are anchored with zero mass.
//  * elements: structure-of-arrays planes (plane k of field f at
//    f + k * Tp), so one warp reads 32 consecutive elements of a plane with
//    one coalesced transaction; each body's elements are padded to TILE.
//  * per-(element, corner) outputs (element force, diagonal block, matvec
//    product) are Vec4 records at index 4 e + c, consumed by a
//    node -> (element, corner) CSR gather in ascending element order: this
//    reproduces the reference's serial scatter order per node
//    (solver.cc:1354-1572, 904-1048) with no floating-point atomics.
//
// Reductions that feed decisions are deterministic: per-tile partial sums in
// FP64 (warp shuffle, then a fixed shared-memory tree), summed over a body's
// tiles in tile order.  Integer counts and flags use integer atomics.
#pragma once

#include "tl_math.cuh"

namespace tl {

constexpr int TILE = 256;  // nodes or elements per tile; one tile per 256-thread block pass

template <class S> struct alignas(4 * sizeof(S)) Vec4 { S x, y, z, w; };

template <class S> __device__ __forceinline__ Vec4<S> ld4(const Vec4<S>* p) { return *p; }
template <class S> __device__ __forceinline__ Vec4<S> ld4cg(const Vec4<S>* p);
template <> __device__ __forceinline__ Vec4<float> ld4cg<float>(const Vec4<float>* p) {
  const float4 v = __ldcg(reinterpret_cast<const float4*>(p));
  return {v.x, v.y, v.z, v.w};
}
template <> __device__ __forceinline__ Vec4<double> ld4cg<double>(const Vec4<double>* p) {
  const double2 a = __ldcg(reinterpret_cast<const double2*>(p));
  const double2 b = __ldcg(reinterpret_cast<const double2*>(p) + 1);
  return {a.x, a.y, b.x, b.y};
}
// Read-only (non-coherent cache) loads of data no kernel writes during the launch.
template <class S> __device__ __forceinline__ Vec4<S> ld4g(const Vec4<S>* p);
template <> __device__ __forceinline__ Vec4<float> ld4g<float>(const Vec4<float>* p) {
  const float4 v = __ldg(reinterpret_cast<const float4*>(p));
  return {v.x, v.y, v.z, v.w};
}
template <> __device__ __forceinline__ Vec4<double> ld4g<double>(const Vec4<double>* p) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(p));
  const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
  return {a.x, a.y, b.x, b.y};
}
template <class S> __device__ __forceinline__ V3<S> xyz(Vec4<S> v) { return {v.x, v.y, v.z}; }
template <class S> __device__ __forceinline__ Vec4<S> pack(V3<S> v, S w = S(0)) { return {v.x, v.y, v.z, w}; }
template <class S, class T> __device__ __forceinline__ Vec4<S> packc(V3<T> v, T w = T(0)) {
  return {S(v.x), S(v.y), S(v.z), S(w)};
}

struct BodyDev {
  uint32_t node_begin, node_end;  // real nodes [begin, end) in global numbering
  uint32_t node_tile_begin, node_tile_end;
  uint32_t elem_begin, elem_end;  // real elements
  uint32_t elem_tile_begin, elem_tile_end;
};

// Per-body generalized-alpha constants of the current step (solver.cc:531-566,
// 3574-3583).  Computed on the host in the system's arithmetic.
struct BodyStepDev {
  uint32_t substeps;  // body takes part in pass p iff p < substeps
  uint32_t limit;     // PCG iteration cap
  uint32_t floating;  // floats (solver.cc:2964-2971): no anchored node, rigid split on
  uint32_t projected; // RigidSplit::Projected: momentum and torque restored each substep
  double inner, carry, alpha_f, alpha_m, beta, gamma;
  double inertia, hstep, scale;  // (1 - alpha_m), h_eff, h_eff^2
  double gx, gy, gz;
  double tolerance;
  double check_inner, check_carry;  // predictor-inversion test at dt / configured
};

// Material lane (material.cc:71-78 with nu clamped to [0, 0.49]); lambda and mu
// are youngs * unit.
struct MatDev {
  double lam_unit, mu_unit, youngs, yield, hardening;
  uint32_t yields, pad;
};

// Per-body accumulators written by kernels (integer atomics) and by the
// finalize kernel (FP64 sums over tiles).
struct BodyAccDev {
  uint32_t nonfinite, grew, inverts, pad;
  unsigned long long min_j_key;  // order-preserving key of the smallest J seen
  unsigned long long moved_key;  // max |increment| (non-negative double bits)
  unsigned long long extent_key; // max |x_evaluated|
  double energy, right_sq, kinetic;
};

struct CgBodyDev {
  double squared, target, floor, length, stride, blend, start_res, rel_res;
  uint32_t taken, done, pad0, pad1;
};

struct CgReportDev {
  uint32_t iterations, capped, applications, solves, tangent_iterations, pad;
  double worst_rel;
  // the current substep's solves (the reference's primaryResult, solver.cc:3919-3950, 4095-4097, 4245):
  // iterations summed, the first solve's start residual, the last solve's end residual
  uint32_t pass_iterations, pass_solves;
  double pass_start, pass_end;
};

// One substep's record of the reference's per-substep report lists
// (StepReport::cgPerSubstep, cgStartResidual, cgEndResidual, solver.h:299-301).
struct SubstepRecordDev {
  uint32_t iterations, pad;
  double start_residual, end_residual;
};
constexpr uint32_t SUBSTEP_RECORDS = 16;  // substeps recorded per body and step

// Floating frame of one body (FloatingFrame, solver.cc:2944-2961), FP64.
// Positions are kept relative to the body's rest centre of mass X0 (fixed at
// creation): `shift` is the current centre minus X0, so a node's arm from the
// centre is (X - X0) + (u - shift) with no large coordinate in it.
struct FrameDev {
  double rest_centre[3];  // X0: mass-weighted rest centre
  double mass;            // total mass
  double shift[3], velocity[3], acceleration[3];
  double next_shift[3], next_velocity[3], next_acceleration[3];
  double momentum[3], torque[3];
  double spin[3], spin_rate[3], weighted_spin[3], weighted_rate[3], end_spin[3], end_rate[3];
  double turn[9];         // row-major end turn of the substep
  double mean[3];         // mass-weighted mean of the solved frame acceleration
  double restore[3], settle[3];
};
constexpr int FRAME_PART = 12;  // per node tile partial sums of the frame moments

struct GridSyncDev {
  unsigned int arrive;
  unsigned int generation;
  int error;
  int active;      // bodies still iterating in the current PCG solve
  int active_odd;  // its copy for odd phases of the one-barrier batched PCG (kPcgBatchSellPipe)
  int pad;
};

// Per-element matvec operator, one record per element: the gradients
// R g_k (corotated) or g_k (SNH), k = 1..3, and the coefficients (a, b, c),
// h_eff^2 V folded in, as (g1x g1y g1z g2x) (g2y g2z g3x g3y) (g3z a b c).
// A record is read whole by one thread, so a gather by element touches 3
// contiguous 16-byte pieces.  The rotated flow normal of the corotated
// consistent tangent, (xx yy zz xy) (xz yz - -), is a separate pair per
// element (Sys::onorm), read only by tangent solves.
template <class S> struct OpRec {
  Vec4<S> q[3];
};

template <class S> struct Sys {
  uint32_t bodies, Vp, Tp, node_tiles, elem_tiles;
  const BodyDev* body;
  const BodyStepDev* step;
  const MatDev* mat;
  const uint32_t* node_tile_body;
  const uint32_t* elem_tile_body;
  // nodes
  const Vec4<S>* rest4;   // (X, Y, Z, mass)
  const uint8_t* anch;
  const Vec4<S>* pres;    // prescribed velocity of anchored nodes
  Vec4<S>* u;             // displacement
  Vec4<S>* v;
  Vec4<S>* a;
  Vec4<S>* carried;
  Vec4<S>* shifted;
  Vec4<S>* weighted;
  Vec4<S>* total;
  Vec4<S>* incr;
  Vec4<S>* right;
  Vec4<S>* pre0;          // block-Jacobi inverse (xx, yy, zz, xy)
  Vec4<S>* pre1;          // (xz, yz, -, -)
  Vec4<S>* r;
  Vec4<S>* z;
  Vec4<S>* p;
  Vec4<S>* ap;            // A p (kPcgBatch); s = A p by recurrence (kPcg1)
  Vec4<S>* w;             // A u (kPcg1)
  const uint32_t* start;  // [Vp + 1]
  const uint32_t* entry;  // 4 e + c, ascending e per node
  // elements
  const uint4* tet;
  const double* dm;       // 9 planes, FP64 Dm^-1 (row-major)
  const S* dms;           // 9 planes, Dm^-1 in S (aliases dm in FP64)
  const double* vold;     // volume (FP64)
  const S* vols;          // volume in S
  const uint32_t* lane;
  const double* eyoung;   // per-element E override or null
  S* op;                  // 9 planes: committed R (corotated) or F (SNH)
  OpRec<S>* orec;         // [Tp] per-element matvec operator records
  S* sell_val;                  // assembled operator's blocks (tl_sell.cuh) or null
  const uint32_t* sell_diag;    // [rows] position of each node row's diagonal block, or null
  Vec4<S>* onorm;         // [2 Tp] rotated flow normal pairs (corotated consistent tangent)
  Vec4<S>* plast;         // 2 planes: (exx, eyy, ezz, exy), (exz, eyz, equivalent, -)
  Vec4<S>* fe;            // [4][Tp] corner planes: (fx, fy, fz, Dxx)
  Vec4<S>* de;            // [4][Tp] (Dyy, Dzz, Dxy, Dxz)
  S* de2;                 // [4][Tp] Dyz
  Vec4<S>* ye;            // [4 Tp] matvec products
  // reductions
  double* part;           // [node_tiles * 4] PCG partials
  double* npart;          // [node_tiles * 2] right^2 (0), kinetic (1)
  double* epart;          // [elem_tiles] elastic energy
  uint32_t* loading;      // [bodies] per assemble: elements past the loading margin
  uint32_t* yielding;     // [bodies] per assemble: elements on the yield surface
  BodyAccDev* acc;
  CgBodyDev* cg;
  CgReportDev* cgrep;
  unsigned int* counter;  // [bodies]
  GridSyncDev* sync;
  // two-level assembly (single-body PCG): per element tile, the distinct nodes
  // it touches ("slots"), with a tile-local CSR of (local element, corner)
  // codes; per node, the slots that hold its partial sums, in tile order.
  const uint2* tile_meta;      // [elem_tiles] (first slot, slot count)
  const uint16_t* tile_off;    // [elem_tiles][4 TILE + 1] offsets into tile_ent
  const uint16_t* tile_ent;    // [elem_tiles][4 TILE] codes 4 * local element + corner
  Vec4<S>* slot_part;          // [slots] tile-local sums of y_e
  const uint32_t* tile_node;   // [slots] global node of each slot
  const uint2* eloc;           // [Tp] an element's 4 corners as slot indices within its tile (4 x u16)
  const uint4* ns_inline;      // [2][Vp] a node's first 8 slot ids (NO_SLOT when unused)
  const uint32_t* ns_start;    // [Vp + 1] slots beyond the first 8 (overflow CSR)
  const uint32_t* ns_slot;     // [overflow slots]
  double* blk_part;            // [3 * grid] per-block partial sums
  uint8_t* yflag;              // [Tp] 1 where the last element pass found the trial state yielding, or null
  // stiffness damping (null when no material of the system damps)
  const S* dtau;               // [Tp] damping weight of each element's lane (0: undamped)
  S* dfit;                     // [20][Tp] rigid fit at the last assemble: arms (12), inverse inertia
                               // (xx, yy, zz, xy, xz, yz), damping coefficients (a, b)
  // finite-strain plastic flow (null unless the system's plasticity is Hencky)
  double* hk;                  // [10][Tp] plastic map P = Fp^-1 (9 planes, row-major), hardening variable
  const double* flim;          // [3 lanes] per material lane: crush stress, crush limit, plastic cap
  // floating bodies (null until a step has a floating body)
  FrameDev* frame;             // [bodies]
  double* fpart;               // [node_tiles][FRAME_PART] frame moment partials
  Vec4<S>* relv;               // frame velocity of each node, then its world arm at the substep end
  Vec4<S>* drive;              // external and fictitious force of each node (replaces m g)
  // per-body gate of a batched plastic Newton round (null: every body takes part): a launch
  // acts on body b only when gate[b] & gate_bit; the low bits carry the body's element-pass mode
  const uint32_t* gate;
  uint32_t gate_bit;
};

// Gate bits (above the ElementMode bits) of the batched Newton rounds.
constexpr uint32_t GATE_ASSEMBLE = 1u << 8;
constexpr uint32_t GATE_ZERO_TOTAL = 1u << 9;
constexpr uint32_t GATE_TOTAL_FROM_LOWEST = 1u << 10;
constexpr uint32_t GATE_BACKTRACK = 1u << 11;
constexpr uint32_t GATE_LOWEST_FROM_TOTAL = 1u << 12;
constexpr uint32_t GATE_INCR_FROM_A = 1u << 13;
constexpr uint32_t GATE_ACCEPT = 1u << 14;
constexpr uint32_t GATE_ADD = 1u << 15;
constexpr uint32_t GATE_A_FROM_TOTAL = 1u << 16;
constexpr uint32_t GATE_ELASTIC = 1u << 17;   // bodies on the three-read elastic path in a Newton batch
constexpr uint32_t GATE_SOLVE0 = 1u << 20;    // + group (x0zero + 2 tangent): the four PCG launch groups

constexpr int TILE_OFF_STRIDE = 4 * TILE + 4;  // 4 TILE + 1 offsets, padded to 8-byte rows

// Position of the (element, corner) record q = 4 e + c in the corner-major
// planes of fe / de / de2 (a warp's stores of one corner are contiguous).
__host__ __device__ __forceinline__ size_t cornerAt(uint32_t q, uint32_t Tp) {
  return size_t(q & 3u) * Tp + (q >> 2);
}
constexpr uint32_t NO_SLOT = 0xffffffffu;

// ------------------------------------------------------------ helpers ----

__device__ __forceinline__ unsigned long long minKey(double v) {
  // order-preserving map double -> uint64 so that atomicMin finds the min
  const unsigned long long b = __double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__host__ __device__ __forceinline__ double fromMinKey(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
#ifdef __CUDA_ARCH__
  return __longlong_as_double(b);
#else
  double d;
  memcpy(&d, &b, 8);
  return d;
#endif
}

// Sum of N doubles over the 256-thread block in a fixed order; result valid
// in thread 0.
template <int N>
__device__ __forceinline__ void blockSum(double (&v)[N]) {
  __shared__ double red[N][8];
#pragma unroll
  for (int k = 0; k < N; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < N; ++k) red[k][warp] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      double s = 0.0;
      for (int w = 0; w < (TILE >> 5); ++w) s += red[k][w];
      v[k] = s;
    }
  }
  __syncthreads();
}

template <class S>
__device__ __forceinline__ V3<double> gradientsOf(const double* dm, uint32_t Tp, uint32_t e, V3<double> g[4]) {
  double d[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) d[k] = __ldg(dm + size_t(k) * Tp + e);
  g[1] = {d[0], d[1], d[2]};
  g[2] = {d[3], d[4], d[5]};
  g[3] = {d[6], d[7], d[8]};
  g[0] = -(g[1] + g[2] + g[3]);  // material.cc:199-207
  return g[0];
}

template <class S> __device__ __forceinline__ void gradientsS(const S* dms, uint32_t Tp, uint32_t e, V3<S> g[4]) {
  S d[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) d[k] = __ldg(dms + size_t(k) * Tp + e);
  g[1] = {d[0], d[1], d[2]};
  g[2] = {d[3], d[4], d[5]};
  g[3] = {d[6], d[7], d[8]};
  g[0] = -(g[1] + g[2] + g[3]);
}

// Symmetric 3x3 stored as (xx, yy, zz, xy, xz, yz).
template <class T> struct Sym { T xx, yy, zz, xy, xz, yz; };
template <class T> __device__ __forceinline__ V3<T> symMul(const Sym<T>& s, V3<T> v) {
  return {s.xx * v.x + s.xy * v.y + s.xz * v.z, s.xy * v.x + s.yy * v.y + s.yz * v.z,
          s.xz * v.x + s.yz * v.y + s.zz * v.z};
}
template <class T> __device__ __forceinline__ T symTrace(const Sym<T>& s) { return s.xx + s.yy + s.zz; }
template <class T> __device__ __forceinline__ T symContract(const Sym<T>& a, const Sym<T>& b) {
  return a.xx * b.xx + a.yy * b.yy + a.zz * b.zz + T(2) * (a.xy * b.xy + a.xz * b.xz + a.yz * b.yz);
}
template <class T> __device__ __forceinline__ Sym<T> symOf(const M3<T>& m) {
  return {m.m[0][0], m.m[1][1], m.m[2][2], T(0.5) * (m.m[0][1] + m.m[1][0]), T(0.5) * (m.m[0][2] + m.m[2][0]),
          T(0.5) * (m.m[1][2] + m.m[2][1])};
}

// Tangent stress of the J2 law (material.cc:636-650) applied to a symmetric
// strain: K tr(e) I + 2 mu theta dev(e) - 2 mu thetaBar (n : e) n.
template <class T>
__device__ __forceinline__ Sym<T> tangentStress(const Sym<T>& e, T bulk, T mu, T theta, T thetaBar, const Sym<T>& n) {
  const T tr = symTrace(e);
  const T third = tr / T(3);
  const T a = T(2) * mu * theta;
  const T ne = T(2) * mu * thetaBar * symContract(n, e);
  Sym<T> s;
  s.xx = bulk * tr + a * (e.xx - third) - ne * n.xx;
  s.yy = bulk * tr + a * (e.yy - third) - ne * n.yy;
  s.zz = bulk * tr + a * (e.zz - third) - ne * n.zz;
  s.xy = a * e.xy - ne * n.xy;
  s.xz = a * e.xz - ne * n.xz;
  s.yz = a * e.yz - ne * n.yz;
  return s;
}

template <class S> __device__ __forceinline__ bool bodyActive(const Sys<S>& s, uint32_t b, uint32_t pass) {
  return pass < s.step[b].substeps && (!s.gate || (s.gate[b] & s.gate_bit) != 0u);
}

__device__ __forceinline__ unsigned long long globalTimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid-wide barrier for a cooperative launch.  Every block arrives once per
// barrier; the last arrival resets the counter and advances the generation.
// Waiting is bounded: after TL_BARRIER_LIMIT_NS the waiting block records
// an error in sync->error and returns false, and so does every block that
// sees the error flag, so a stalled grid ends instead of hanging.
#define TL_BARRIER_LIMIT_NS 2000000000ull
__device__ __forceinline__ bool gridBarrier(GridSyncDev* sync) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int good = 1;
    volatile unsigned int* gen = &sync->generation;
    const unsigned int seen = *gen;
    __threadfence();
    const unsigned int prev = atomicAdd(&sync->arrive, 1u);
    if (prev == gridDim.x - 1) {
      atomicExch(&sync->arrive, 0u);
      __threadfence();
      atomicAdd(&sync->generation, 1u);
    } else {
      const unsigned long long t0 = globalTimer();
      while (*gen == seen) {
        if (*(volatile int*)&sync->error != 0) {
          good = 0;
          break;
        }
        __nanosleep(32);
        if (globalTimer() - t0 > TL_BARRIER_LIMIT_NS) {
          atomicExch(&sync->error, 5);  // TL_ERR_TIMEOUT
          good = 0;
          break;
        }
      }
    }
    __threadfence();
    ok = good && (*(volatile int*)&sync->error == 0);
  }
  __syncthreads();
  return ok != 0;
}

// Returns true in the block that processed the last tile of body b in this
// phase (the tile's partials must already be written by thread 0).
__device__ __forceinline__ bool lastTileOfBody(unsigned int* counter, uint32_t ntiles) {
  __shared__ int last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int prev = atomicAdd(counter, 1u);
    last = prev == ntiles - 1u;
    if (last) {
      atomicExch(counter, 0u);
      __threadfence();
    }
  }
  __syncthreads();
  return last != 0;
}

// Fixed-order sum of field k of the partials of tiles [t0, t1).  Block-wide;
// result valid in thread 0.
template <int N>
__device__ __forceinline__ void sumTiles(const double* part, uint32_t t0, uint32_t t1, double (&out)[N]) {
#pragma unroll
  for (int k = 0; k < N; ++k) out[k] = 0.0;
  for (uint32_t t = t0 + threadIdx.x; t < t1; t += TILE)
#pragma unroll
    for (int k = 0; k < N; ++k) out[k] += __ldcg(part + size_t(t) * 4 + k);
  blockSum<N>(out);
}

// Block-wide integer sums (one atomic per block instead of one per thread).
__device__ __forceinline__ uint32_t blockCount(bool flag) {
  __shared__ uint32_t cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  const uint32_t w = __popc(__ballot_sync(0xffffffffu, flag));
  if ((threadIdx.x & 31) == 0 && w) atomicAdd(&cnt, w);
  __syncthreads();
  const uint32_t r = cnt;
  __syncthreads();
  return r;
}
// Block-wide max of 64-bit keys; result valid in thread 0.
__device__ __forceinline__ unsigned long long blockMaxKey(unsigned long long k) {
  __shared__ unsigned long long red[TILE / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long q = __shfl_down_sync(0xffffffffu, k, o);
    k = q > k ? q : k;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = k;
  __syncthreads();
  if (threadIdx.x == 0)
    for (int w = 1; w < TILE / 32; ++w) k = red[w] > k ? red[w] : k;
  __syncthreads();
  return k;
}

// Asynchronous global -> shared copies (cp.async, 4, 8 or 16 bytes; 16-byte
// copies bypass L1).  Both addresses must be aligned to the copy size.
template <int N> __device__ __forceinline__ void cpAsync(void* dst, const void* src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  if constexpr (N == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(src), "n"(N) : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cpAsyncWaitAll() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// ------------------------------------------------------------- kernels ----

// Predictor (solver.cc:3691-3700): carried = a; shifted = u + h v + (1/2 - beta) h^2 a;
// weighted = (1 - alpha_f) shifted + alpha_f u.
template <class S>
__global__ void __launch_bounds__(TILE) kPredict(Sys<S> s, uint32_t pass) {
  const uint32_t tile = blockIdx.x, b = s.node_tile_body[tile];
  if (!bodyActive(s, b, pass)) return;
  const uint32_t n = tile * TILE + threadIdx.x;
  if (n >= s.body[b].node_end) return;
  const BodyStepDev& st = s.step[b];
  const V3<double> u = cvt<double>(xyz(s.u[n])), v = cvt<double>(xyz(s.v[n])), a = cvt<double>(xyz(s.a[n]));
  if (st.floating) {
    // solver.cc:3662-3690 in the frame of the body's centre and spin.  Frame
    // positions are kept as displacements from the rest arm X - X0: uf = u - shift.
    const FrameDev& f = s.frame[b];
    const V3<double> rest = cvt<double>(xyz(s.rest4[n]));
    const V3<double> restArm = rest - V3<double>{f.rest_centre[0], f.rest_centre[1], f.rest_centre[2]};
    const V3<double> uf = u - V3<double>{f.shift[0], f.shift[1], f.shift[2]};
    const V3<double> arm = restArm + uf;
    const V3<double> spin = {f.spin[0], f.spin[1], f.spin[2]};
    const V3<double> moving = v - V3<double>{f.velocity[0], f.velocity[1], f.velocity[2]} - cross(spin, arm);
    const V3<double> turning = a - V3<double>{f.acceleration[0], f.acceleration[1], f.acceleration[2]} -
                               cross(V3<double>{f.spin_rate[0], f.spin_rate[1], f.spin_rate[2]}, arm) -
                               cross(spin, cross(spin, arm)) - 2.0 * cross(spin, moving);
    const V3<double> sh = uf + st.inner * moving + st.carry * turning;
    const V3<double> w = (1.0 - st.alpha_f) * sh + st.alpha_f * uf;
    const V3<double> at = restArm + w;  // the reference's weighted frame position
    const V3<double> held = {f.weighted_spin[0], f.weighted_spin[1], f.weighted_spin[2]};
    const V3<double> rate = {f.weighted_rate[0], f.weighted_rate[1], f.weighted_rate[2]};
    const double lag = (1.0 - st.alpha_f) * (1.0 - st.gamma) * st.inner;
    const double mass = double(s.rest4[n].w);
    const V3<double> drive =
        -mass * (cross(held, cross(held, at)) + cross(rate, at) + 2.0 * cross(held, moving + lag * turning));
    s.relv[n] = packc<S>(moving);
    s.carried[n] = packc<S>(turning);
    s.shifted[n] = packc<S>(sh);
    s.weighted[n] = packc<S>(w);
    s.drive[n] = packc<S>(drive);
    s.a[n] = packc<S>(turning);
    return;
  }
  const V3<double> sh = u + st.inner * v + st.carry * a;
  const V3<double> w = (1.0 - st.alpha_f) * sh + st.alpha_f * u;
  s.carried[n] = s.a[n];
  s.shifted[n] = packc<S>(sh);
  s.weighted[n] = packc<S>(w);
}

// predictorInverts (solver.cc:568-623): does any tet of the body invert at the
// predicted weighted position for h = dt / configured?
template <class S>
__global__ void __launch_bounds__(TILE) kInversionCheck(Sys<S> s) {
  const uint32_t tile = blockIdx.x, b = s.elem_tile_body[tile];
  const uint32_t e = tile * TILE + threadIdx.x;
  if (e >= s.body[b].elem_end) return;
  const BodyStepDev& st = s.step[b];
  if (st.floating) return;  // a floating body is not tested (solver.cc:3574-3583)
  const uint4 t = __ldg(&s.tet[e]);
  const uint32_t nodes[4] = {t.x, t.y, t.z, t.w};
  V3<double> g[4];
  gradientsOf<S>(s.dm, s.Tp, e, g);
  M3<double> h = zero3<double>();
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const uint32_t n = nodes[c];
    const V3<double> u = cvt<double>(xyz(s.u[n])), v = cvt<double>(xyz(s.v[n])), a = cvt<double>(xyz(s.a[n]));
    const V3<double> sh = u + st.check_inner * v + st.check_carry * a;
    addOuter(h, (1.0 - st.alpha_f) * sh + st.alpha_f * u, g[c]);
  }
  if (!(1.0 + volumeChange(h) > 0.0)) atomicOr(&s.acc[b].inverts, 1u);
}

enum ElementMode : uint32_t {
  EM_KEEP = 1u,        // store the trial plastic point (assembleElastic's `keep`)
  EM_CONSISTENT = 2u,  // scratch.stiffness is the consistent tangent (bindStiffness(true))
  EM_MAPPING = 4u,     // returnMapping
  EM_COMMIT = 8u,      // commitPlastic: plastic point only, no forces
  EM_YIELDING = 16u,   // some lane of the system yields: stage the plastic points
};

// One element tile's inputs in shared memory, filled by cp.async when the
// element pass starts: one wave of coalesced copies per tile instead of
// loads spread through the kernel, and the second read of Dm^-1 and the
// plastic point (after the rotation) come from here, not from L2.
// The displacement gradient H is parked here across the corotated law's
// rotation: the rotation's FP64 iteration needs every register it can get,
// and values that spill instead go to local memory, which shares the L1
// with this stage and misses it.
template <class S> struct ElementStage {
  double dm[9][TILE];       // Dm^-1 planes (FP64)
  double h[9][TILE];        // H (row-major planes) while the rotation runs
  double vol[TILE];
  uint4 tet[TILE];
  Vec4<S> plast[2][TILE];
  uint32_t lane[TILE];
};
// Dynamic shared memory of kElement (above the 48 KB a launch gets without
// opting in; the host raises the limit once per instantiation).
template <class S> constexpr size_t elementStageBytes() { return sizeof(ElementStage<S>); }

// Element pass (assembleElastic, solver.cc:1354-1572; trial material.cc:236-265;
// tetPointTrial material.cc:978-1057; SNH neohookean.cc:41-47, 183-192).
// Kinematics and the law run in FP64 whatever S is; outputs are stored in S.
// Positions are base + reach * dir (the reference's `evaluated`), in
// displacement form.
// Resident 256-thread blocks per SM the element pass is compiled for: three
// for the FP32-mixed corotated pass (80 registers; 4% less time per launch on
// the 393,216-tet plastic block than two blocks at 128 registers, with
// bitwise the same results), two for the others (the FP64 pass keeps its
// 128 registers).
template <class S, int LAW> constexpr int elementMinBlocks() {
  return std::is_same_v<S, float> && LAW == 0 ? 3 : 2;
}
// HK: the corotated law from each tet's plastic rest shape (finite-strain
// flow): F' = F P, gradients g' = P^T g, volume V / det P, where P = Fp^-1 is
// the tet's plastic map (plasticRest, plasticflow.cc:263-300: Dm' = Fp Dm,
// V' = V det Fp); the small-strain return map is off.
template <class S, int LAW, bool HK>
__device__ __forceinline__ void elementTile(const Sys<S>& s, const Vec4<S>* base, const Vec4<S>* dir, uint32_t pass,
                                            uint32_t mode, double margin, uint32_t tile) {
  static_assert(!HK || LAW == 0, "the plastic rest shape is written for the corotated law");
  const uint32_t b = s.elem_tile_body[tile];
  if (!bodyActive(s, b, pass)) return;
  if (s.gate)  // a batched Newton round: the body's own mapping and tangent choice
    mode = (mode & ~uint32_t(EM_CONSISTENT | EM_MAPPING)) | (s.gate[b] & uint32_t(EM_CONSISTENT | EM_MAPPING));
  const uint32_t e = tile * TILE + threadIdx.x;
  const bool valid = e < s.body[b].elem_end;
  extern __shared__ __align__(32) unsigned char tlElementStage[];
  ElementStage<S>& stage = *reinterpret_cast<ElementStage<S>*>(tlElementStage);
  const uint32_t me = threadIdx.x;
  if (valid) {
    cpAsync<16>(&stage.tet[me], &s.tet[e]);
#pragma unroll
    for (int k = 0; k < 9; ++k) cpAsync<8>(&stage.dm[k][me], s.dm + size_t(k) * s.Tp + e);
    cpAsync<8>(&stage.vol[me], s.vold + e);
    cpAsync<4>(&stage.lane[me], s.lane + e);
    if (LAW == 0 && !HK && (mode & EM_YIELDING)) {
#pragma unroll
      for (int k = 0; k < 2; ++k)
#pragma unroll
        for (int h = 0; h < int(sizeof(Vec4<S>)) / 16; ++h)
          cpAsync<16>(reinterpret_cast<unsigned char*>(&stage.plast[k][me]) + 16 * h,
                      reinterpret_cast<const unsigned char*>(&s.plast[size_t(k) * s.Tp + e]) + 16 * h);
    }
  }
  cpAsyncCommit();
  cpAsyncWaitAll();
  __syncthreads();
  const auto stagedGradients = [&](V3<double> g[4]) {
    g[1] = {stage.dm[0][me], stage.dm[1][me], stage.dm[2][me]};
    g[2] = {stage.dm[3][me], stage.dm[4][me], stage.dm[5][me]};
    g[3] = {stage.dm[6][me], stage.dm[7][me], stage.dm[8][me]};
    g[0] = -(g[1] + g[2] + g[3]);  // material.cc:199-207
  };
  double energy = 0.0;
  bool isLoading = false, isYielding = false, grew = false, nonfinite = false;
  unsigned long long jkey = ~0ull;
  if (valid) {
    const BodyStepDev& st = s.step[b];
    const double reach = dir ? st.scale : 0.0;
    const uint4 t = stage.tet[me];
    const uint32_t nodes[4] = {t.x, t.y, t.z, t.w};
    M3<double> H = zero3<double>();  // displacement gradient, F = I + H
    {
      V3<double> g0[4];
      stagedGradients(g0);
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const uint32_t n = nodes[c];
        V3<double> uu = cvt<double>(xyz(base[n]));
        if (dir) uu = uu + reach * cvt<double>(xyz(dir[n]));
        addOuter(H, uu, g0[c]);
      }
    }
    double vol = stage.vol[me];
    if constexpr (HK) {  // H' = (I + H) P - I
      M3<double> P;
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) P.m[i][j] = s.hk[size_t(3 * i + j) * s.Tp + e];
      M3<double> F = H;
      F.m[0][0] += 1.0;
      F.m[1][1] += 1.0;
      F.m[2][2] += 1.0;
      H = mul(F, P);
      H.m[0][0] -= 1.0;
      H.m[1][1] -= 1.0;
      H.m[2][2] -= 1.0;
      vol /= det3(P);
    }
    const MatDev m = s.mat[stage.lane[me]];
    const double youngs = s.eyoung ? s.eyoung[e] : m.youngs;
    const double lam = youngs * m.lam_unit, mu = youngs * m.mu_unit;
    const double change = volumeChange(H);
    jkey = minKey(1.0 + change);
    bool finite = true;
    // per-corner force and diagonal block, stored as soon as they are formed
    // (forces in FP64; the diagonal blocks, like the matvec operator, are formed
    // in the storage type S: they only precondition and are stored as S)
    auto emit = [&](int c, const V3<S>& f, const Sym<S>& d) {
      finite = finite && isfinite(f.x) && isfinite(f.y) && isfinite(f.z);
      const size_t at = size_t(c) * s.Tp + e;
      s.fe[at] = Vec4<S>{S(f.x), S(f.y), S(f.z), S(d.xx)};
      s.de[at] = Vec4<S>{S(d.yy), S(d.zz), S(d.xy), S(d.xz)};
      s.de2[at] = S(d.yz);
    };
    if (LAW == 0) {
      M3<double> F = H;
      F.m[0][0] += 1.0;
      F.m[1][1] += 1.0;
      F.m[2][2] += 1.0;
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) stage.h[3 * i + j][me] = H.m[i][j];
      // ElementRotation::Polar for floating bodies, Invertible otherwise (solver.cc:3587-3588)
      const M3<double> R = elementRotation(F, st.floating == 0u);
      // H comes back from shared memory (the clobber keeps the compiler from
      // holding it in registers through the rotation instead)
      asm volatile("" ::: "memory");
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) H.m[i][j] = stage.h[3 * i + j][me];
      // Corotated strain (material.cc:92-109, 155-161): the offsets
      // R^T (x_c - x_mean) - (X_c - X_mean) summed against g_c.  Because
      // sum_c g_c = 0 and sum_c X_c g_c^T = Ds Dm^-1 = I, that sum is
      // R^T F - I = R^T H + (R^T - I), formed here without the rest positions.
      M3<double> D = mul(transpose(R), H);
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) D.m[i][j] += R.m[j][i] - (i == j ? 1.0 : 0.0);
      const Sym<double> eps = symOf(D);
      // the rotation in S from here on (the committed rotation is stored in S)
      M3<S> Rw;
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Rw.m[i][j] = S(R.m[i][j]);
      if (!(mode & EM_COMMIT))
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) s.op[size_t(3 * i + j) * s.Tp + e] = Rw.m[i][j];
      // From here on the arithmetic is the storage type S: the strain above
      // needs FP64 (it is a small difference of O(1) quantities); the return
      // map, stress and forces only need the relative accuracy of the S
      // records they end in.  In FP64 systems nothing changes.
      using C = S;
      const bool yields = !HK && m.yields != 0u;
      const C lamC = C(lam), muC = C(mu), volC = C(vol);
      const C bulk = C(lam + 2.0 * mu / 3.0);
      Sym<C> stress;
      C theta = C(1), thetaBar = C(0);
      Sym<C> normal = {0, 0, 0, 0, 0, 0};
      if (yields) {
        // returnMap (material.cc:594-634)
        const Vec4<S> p0 = stage.plast[0][me], p1 = stage.plast[1][me];
        const Sym<C> ep = {C(p0.x), C(p0.y), C(p0.z), C(p0.w), C(p1.x), C(p1.y)};
        const C eq = C(p1.z);
        const Sym<C> el = {C(eps.xx - double(p0.x)), C(eps.yy - double(p0.y)), C(eps.zz - double(p0.z)),
                           C(eps.xy - double(p0.w)), C(eps.xz - double(p1.x)), C(eps.yz - double(p1.y))};
        const C pressure = bulk * symTrace(el);
        const C third = symTrace(el) / C(3);
        const C twoMu = C(2) * muC;
        const Sym<C> tr = {twoMu * (el.xx - third), twoMu * (el.yy - third), twoMu * (el.zz - third),
                           twoMu * el.xy, twoMu * el.xz, twoMu * el.yz};
        const C norm = sqrt(symContract(tr, tr));
        const C equivalent = C(sqrt(1.5)) * norm;
        const C hard = C(fmax(m.hardening, 0.0));
        const C radius = C(m.yield) + hard * eq;
        Sym<C> next = ep;
        C nextEq = eq;
        C excess = C(0);
        if (!(mode & EM_MAPPING) || !(equivalent > radius) || !(norm > C(0))) {
          stress = {tr.xx + pressure, tr.yy + pressure, tr.zz + pressure, tr.xy, tr.xz, tr.yz};
        } else {
          const C gamma = (equivalent - radius) / (C(3) * muC + hard);
          const C inv = C(1) / norm;
          const Sym<C> n = {tr.xx * inv, tr.yy * inv, tr.zz * inv, tr.xy * inv, tr.xz * inv, tr.yz * inv};
          const C th = C(1) - C(3) * muC * gamma / equivalent;
          stress = {th * tr.xx + pressure, th * tr.yy + pressure, th * tr.zz + pressure, th * tr.xy, th * tr.xz,
                    th * tr.yz};
          excess = (equivalent - radius) / radius;
          const C sg = C(sqrt(1.5)) * gamma;
          next = {ep.xx + sg * n.xx, ep.yy + sg * n.yy, ep.zz + sg * n.zz,
                  ep.xy + sg * n.xy, ep.xz + sg * n.xz, ep.yz + sg * n.yz};
          nextEq = eq + gamma;
          const bool loading = double(excess) > margin;
          if (loading) {  // linearized = response (material.cc:1016-1017)
            theta = th;
            thetaBar = C(3) * muC / (C(3) * muC + hard) - (C(1) - th);
            normal = n;
          }
          isLoading = loading;
          isYielding = true;
        }
        const Sym<C> rem = {C(eps.xx - double(next.xx)), C(eps.yy - double(next.yy)), C(eps.zz - double(next.zz)),
                            C(eps.xy - double(next.xy)), C(eps.xz - double(next.xz)), C(eps.yz - double(next.yz))};
        energy = double(volC * C(0.5) * symContract(stress, rem));
        if ((mode & (EM_KEEP | EM_COMMIT)) != 0u) {
          grew = nextEq > eq;
          s.plast[e] = Vec4<S>{S(next.xx), S(next.yy), S(next.zz), S(next.xy)};
          s.plast[s.Tp + e] = Vec4<S>{S(next.xz), S(next.yz), S(nextEq), S(0)};
        }
      } else {
        const Sym<C> ec = {C(eps.xx), C(eps.yy), C(eps.zz), C(eps.xy), C(eps.xz), C(eps.yz)};
        const C tr = symTrace(ec);
        stress = {lamC * tr + C(2) * muC * ec.xx, lamC * tr + C(2) * muC * ec.yy, lamC * tr + C(2) * muC * ec.zz,
                  C(2) * muC * ec.xy, C(2) * muC * ec.xz, C(2) * muC * ec.yz};
        energy = double(volC * C(0.5) * symContract(stress, ec));
      }
      if (!(mode & EM_COMMIT)) {
        // The gradients are loaded again here rather than kept live through the
        // rotation and the return map; the empty asm keeps the compiler from
        // merging the loads with the first ones.
        asm volatile("" ::: "memory");
        V3<double> g[4];
        {
          g[1] = {stage.dm[0][me], stage.dm[1][me], stage.dm[2][me]};
          g[2] = {stage.dm[3][me], stage.dm[4][me], stage.dm[5][me]};
          g[3] = {stage.dm[6][me], stage.dm[7][me], stage.dm[8][me]};
          if constexpr (HK) {  // g' = P^T g (P reloaded: not kept live through the rotation)
            double p[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) p[k] = s.hk[size_t(k) * s.Tp + e];
#pragma unroll
            for (int c = 1; c < 4; ++c)
              g[c] = {p[0] * g[c].x + p[3] * g[c].y + p[6] * g[c].z, p[1] * g[c].x + p[4] * g[c].y + p[7] * g[c].z,
                      p[2] * g[c].x + p[5] * g[c].y + p[8] * g[c].z};
          }
          g[0] = -(g[1] + g[2] + g[3]);
        }
        const bool tangentDiag = (mode & EM_CONSISTENT) && yields;
        const C th = tangentDiag ? theta : C(1);
        const C thb = tangentDiag ? thetaBar : C(0);
        const Sym<S> nw = normal;
        const S k1 = volC * (bulk + muC * th / C(3)), kmu = volC * muC * th, k3 = -volC * C(2) * muC * thb;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          // R K_cc R^T with K_cc = V[(K + mu theta/3) g g^T + mu theta |g|^2 I - 2 mu thetaBar (n g)(n g)^T]
          const V3<S> gc = cvt<S>(g[c]);
          const V3<S> force = -(volC * mul(Rw, symMul(stress, gc)));  // material.cc:1019-1027
          const V3<S> rg = mul(Rw, gc);
          const V3<S> rn = mul(Rw, symMul(nw, gc));
          const S k2 = kmu * dot(gc, gc);
          emit(c, force, {k1 * rg.x * rg.x + k2 + k3 * rn.x * rn.x, k1 * rg.y * rg.y + k2 + k3 * rn.y * rn.y,
                          k1 * rg.z * rg.z + k2 + k3 * rn.z * rn.z, k1 * rg.x * rg.y + k3 * rn.x * rn.y,
                          k1 * rg.x * rg.z + k3 * rn.x * rn.z, k1 * rg.y * rg.z + k3 * rn.y * rn.z});
        }
        // Matvec operator in the rotated frame: R K R^T p = sum over corners of
        // V sigma_t(sym(sum_b p_b gh_b^T)) gh_a with gh = R g and the rotated
        // normal R n R^T; h_eff^2 V folded into the coefficients.
        const double sv = st.scale * vol;
        const V3<S> gh1 = mul(Rw, cvt<S>(g[1])), gh2 = mul(Rw, cvt<S>(g[2])), gh3 = mul(Rw, cvt<S>(g[3]));
        OpRec<S>& rec = s.orec[e];
        rec.q[0] = Vec4<S>{gh1.x, gh1.y, gh1.z, gh2.x};
        rec.q[1] = Vec4<S>{gh2.y, gh2.z, gh3.x, gh3.y};
        rec.q[2] = Vec4<S>{gh3.z, S(sv * (bulk - 2.0 * mu * th / 3.0)), S(sv * 2.0 * mu * th), S(sv * 2.0 * mu * thb)};
        if (mode & EM_CONSISTENT) {
          M3<S> nm;
          nm.m[0][0] = nw.xx; nm.m[1][1] = nw.yy; nm.m[2][2] = nw.zz;
          nm.m[0][1] = nm.m[1][0] = nw.xy;
          nm.m[0][2] = nm.m[2][0] = nw.xz;
          nm.m[1][2] = nm.m[2][1] = nw.yz;
          const M3<S> nh = mul(mul(Rw, nm), transpose(Rw));
          s.onorm[2 * size_t(e)] = Vec4<S>{nh.m[0][0], nh.m[1][1], nh.m[2][2], nh.m[0][1]};
          s.onorm[2 * size_t(e) + 1] = Vec4<S>{nh.m[0][2], nh.m[1][2], S(0), S(0)};
        }
      }
    } else {
      V3<double> g[4];
      stagedGradients(g);
      // SNH: P = mu (H + H^T - tr H I - cof H) + (lambda + mu)(J - 1) cof F
      M3<double> F = H;
      F.m[0][0] += 1.0;
      F.m[1][1] += 1.0;
      F.m[2][2] += 1.0;
      const M3<double> C = cofactor(F), CH = cofactor(H);
      const double shifted = lam + mu;
      const double trH = trace3(H);
      M3<double> P;
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
          P.m[i][j] = mu * (H.m[i][j] + H.m[j][i] - (i == j ? trH : 0.0) - CH.m[i][j]) + shifted * change * C.m[i][j];
      const double squared = contract(H, H);
      energy = vol * (0.5 * mu * squared - mu * (change - trH) + 0.5 * shifted * change * change);
      if (!(mode & EM_COMMIT)) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const V3<S> bb = cvt<S>(mul(C, g[c]));
          const S k2 = S(vol * mu * dot(g[c], g[c])), k1 = S(vol * shifted);
          emit(c, cvt<S>(-(vol * mul(P, g[c]))), {k1 * bb.x * bb.x + k2, k1 * bb.y * bb.y + k2, k1 * bb.z * bb.z + k2,
                                          k1 * bb.x * bb.y, k1 * bb.x * bb.z, k1 * bb.y * bb.z});
        }
      }
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) s.op[size_t(3 * i + j) * s.Tp + e] = S(F.m[i][j]);
      // Matvec operator: dP = mu dF + ((lambda + mu)(J - 1) - mu) dcof + (lambda + mu)(cof : dF) cof,
      // h_eff^2 V folded into the coefficients; unrotated gradients.
      const double sv = st.scale * vol;
      OpRec<S>& rec = s.orec[e];
      rec.q[0] = Vec4<S>{S(g[1].x), S(g[1].y), S(g[1].z), S(g[2].x)};
      rec.q[1] = Vec4<S>{S(g[2].y), S(g[2].z), S(g[3].x), S(g[3].y)};
      rec.q[2] = Vec4<S>{S(g[3].z), S(sv * mu), S(sv * (shifted * change - mu)), S(sv * shifted)};
    }
    if (!(mode & EM_COMMIT)) nonfinite = !finite;
  }
  if (valid && s.yflag && !(mode & EM_COMMIT)) s.yflag[e] = isYielding ? 1u : 0u;
  // All per-tile results in one fixed-order block reduction (one barrier):
  // counts by warp ballots, the smallest J key and the energy by shuffles,
  // then warps in order in thread 0.
  __shared__ double redEnergy[TILE / 32];
  __shared__ unsigned long long redKey[TILE / 32];
  __shared__ uint32_t redCount[TILE / 32][4];
  const unsigned full = 0xffffffffu;
  const uint32_t c0 = __popc(__ballot_sync(full, isLoading)), c1 = __popc(__ballot_sync(full, isYielding));
  const uint32_t c2 = __popc(__ballot_sync(full, grew)), c3 = __popc(__ballot_sync(full, nonfinite));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    energy += __shfl_down_sync(full, energy, o);
    const unsigned long long q = __shfl_down_sync(full, jkey, o);
    jkey = q < jkey ? q : jkey;
  }
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    redEnergy[warp] = energy;
    redKey[warp] = jkey;
    redCount[warp][0] = c0;
    redCount[warp][1] = c1;
    redCount[warp][2] = c2;
    redCount[warp][3] = c3;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  double sum = 0.0;
  unsigned long long jmin = ~0ull;
  uint32_t nLoading = 0, nYielding = 0, nGrew = 0, nBad = 0;
  for (int w = 0; w < TILE / 32; ++w) {
    sum += redEnergy[w];
    jmin = redKey[w] < jmin ? redKey[w] : jmin;
    nLoading += redCount[w][0];
    nYielding += redCount[w][1];
    nGrew += redCount[w][2];
    nBad += redCount[w][3];
  }
  if (mode & EM_COMMIT) {
    if (nGrew) atomicOr(&s.acc[b].grew, 1u);
    return;
  }
  if (nLoading) atomicAdd(&s.loading[b], nLoading);
  if (nYielding) atomicAdd(&s.yielding[b], nYielding);
  if (nBad) atomicOr(&s.acc[b].nonfinite, 1u);
  atomicMin(&s.acc[b].min_j_key, jmin);
  s.epart[tile] = sum;
}

// The element pass over tiles blockIdx.x, blockIdx.x + gridDim.x, ...: a grid
// of one block per tile, or a resident grid that walks the tiles (no block
// launches between rounds); each tile is worked the same way either way.
template <class S, int LAW, bool HK = false>
__global__ void __launch_bounds__(TILE, elementMinBlocks<S, LAW>())
    kElement(Sys<S> s, const Vec4<S>* base, const Vec4<S>* dir, uint32_t pass, uint32_t mode, double margin) {
  for (uint32_t tile = blockIdx.x; tile < s.elem_tiles; tile += gridDim.x) {
    elementTile<S, LAW, HK>(s, base, dir, pass, mode, margin, tile);
    __syncthreads();  // the stage and the reduction arrays are reused by the next tile
  }
}

// Node gather + balance (solver.cc:3746-3806) + guardPreconditioner
// (solver.cc:1574-1593).  taken: the acceleration the right side subtracts
// (null for the first read).
template <class S>
__global__ void __launch_bounds__(TILE) kNodeAssemble(Sys<S> s, const Vec4<S>* taken, uint32_t pass) {
  const uint32_t tile = blockIdx.x, b = s.node_tile_body[tile];
  if (!bodyActive(s, b, pass)) return;
  const uint32_t n = tile * TILE + threadIdx.x;
  double rr = 0.0;
  if (n < s.body[b].node_end) {
    const BodyStepDev& st = s.step[b];
    const S scale = S(st.scale);
    double f[3] = {0, 0, 0};
    S d[6] = {0, 0, 0, 0, 0, 0};
    const uint32_t k0 = s.start[n], k1 = s.start[n + 1];
    for (uint32_t k = k0; k < k1; ++k) {
      const uint32_t q = __ldg(&s.entry[k]);
      const size_t at = cornerAt(q, s.Tp);
      const Vec4<S> a = s.fe[at], c = s.de[at];
      const S c2 = s.de2[at];
      f[0] += double(a.x);
      f[1] += double(a.y);
      f[2] += double(a.z);
      d[0] += scale * a.w;
      d[1] += scale * c.x;
      d[2] += scale * c.y;
      d[3] += scale * c.z;
      d[4] += scale * c.w;
      d[5] += scale * c2;
    }
    const Vec4<S> rest = ld4g(&s.rest4[n]);
    if (s.anch[n]) {
      if (s.sell_diag) {  // anchored rows of the assembled operator are zero
        S* v = s.sell_val + size_t(s.sell_diag[n] >> 5) * 9 * 32 + (s.sell_diag[n] & 31u);
#pragma unroll
        for (int c = 0; c < 9; ++c) v[c * 32] = S(0);
      }
      s.v[n] = s.pres[n];
      s.a[n] = Vec4<S>{0, 0, 0, 0};
      s.right[n] = Vec4<S>{0, 0, 0, 0};
      s.pre0[n] = Vec4<S>{1, 1, 1, 0};
      s.pre1[n] = Vec4<S>{0, 0, 0, 0};
    } else {
      const double mass = double(rest.w);
      const V3<double> car = cvt<double>(xyz(s.carried[n]));
      // the drive: m g, or the frame's forces for a floating body (solver.cc:3683-3699)
      const V3<double> drive = st.floating ? cvt<double>(xyz(s.drive[n])) : V3<double>{mass * st.gx, mass * st.gy,
                                                                                        mass * st.gz};
      V3<double> rhs = {f[0] + drive.x - st.alpha_m * mass * car.x, f[1] + drive.y - st.alpha_m * mass * car.y,
                        f[2] + drive.z - st.alpha_m * mass * car.z};
      if (taken) rhs = rhs - (st.inertia * mass) * cvt<double>(xyz(taken[n]));
      s.right[n] = packc<S>(rhs);
      rr = dot(rhs, rhs);
      const S im = S(st.inertia * mass);
      const S xx = d[0] + im, yy = d[1] + im, zz = d[2] + im, xy = d[3], xz = d[4], yz = d[5];
      if (s.sell_diag) {  // the assembled operator's diagonal block is this one
        S* v = s.sell_val + size_t(s.sell_diag[n] >> 5) * 9 * 32 + (s.sell_diag[n] & 31u);
        const S m[9] = {xx, xy, xz, xy, yy, yz, xz, yz, zz};
#pragma unroll
        for (int c = 0; c < 9; ++c) v[c * 32] = m[c];
      }
      // inverse of the symmetric block, identity unless det > 0
      const S cxx = yy * zz - yz * yz, cxy = xz * yz - xy * zz, cxz = xy * yz - xz * yy;
      const S det = xx * cxx + xy * cxy + xz * cxz;
      if (det > S(0)) {
        const S inv = S(1) / det;
        s.pre0[n] = Vec4<S>{cxx * inv, (xx * zz - xz * xz) * inv, (xx * yy - xy * xy) * inv, cxy * inv};
        s.pre1[n] = Vec4<S>{cxz * inv, (xy * xz - xx * yz) * inv, 0, 0};
      } else {
        s.pre0[n] = Vec4<S>{1, 1, 1, 0};
        s.pre1[n] = Vec4<S>{0, 0, 0, 0};
      }
    }
  }
  const uint32_t nBad = blockCount(!isfinite(rr));
  if (threadIdx.x == 0 && nBad) atomicOr(&s.acc[b].nonfinite, 1u);
  double v[1] = {rr};
  blockSum<1>(v);
  if (threadIdx.x == 0) s.npart[size_t(tile) * 2] = v[0];
}

// Sum the per-tile partials of each body (one block per body) in tile order.
// which: 0 = elastic energy (element tiles), 1 = right^2, 2 = kinetic (node tiles).
static __global__ void __launch_bounds__(TILE) kFinalize(const BodyDev* body, const double* epart, const double* npart,
                                                  BodyAccDev* acc, uint32_t which) {
  const uint32_t b = blockIdx.x;
  const uint32_t t0 = which == 0 ? body[b].elem_tile_begin : body[b].node_tile_begin;
  const uint32_t t1 = which == 0 ? body[b].elem_tile_end : body[b].node_tile_end;
  double out[1] = {0.0};
  for (uint32_t t = t0 + threadIdx.x; t < t1; t += TILE)
    out[0] += which == 0 ? epart[t] : npart[size_t(t) * 2 + (which - 1)];
  blockSum<1>(out);
  if (threadIdx.x == 0) {
    if (which == 0) acc[b].energy = out[0];
    else if (which == 1) acc[b].right_sq = out[0];
    else acc[b].kinetic = out[0];
  }
}

// ------------------------------------------------------- stiffness damping ----
// D(p) = Pi R K R^T Pi p per damped element (factor.cc:780-853): Pi removes the
// rigid motion fitted to the corners (mean translation and the spin
// I^-1 sum a x p about the centroid), K is the element's elastic stiffness
// (the blocks of tetStiffness, material.cc:209-234) and R its committed
// rotation.  The system operator gains (1 - alpha_f) gamma h tau D, the right
// side loses tau D(v + lag ((1 - gamma) a_prev + gamma a)), lag = (1 - alpha_f) h
// (solver.cc:1006-1007, 3747-3778), and the block-Jacobi diagonal gains the
// corner blocks of (1 - alpha_f) gamma h tau D (solver.cc:755-830).

template <class T>
__device__ __forceinline__ void removeRigid(const V3<T> arm[4], const Sym<T>& inv, V3<T> v[4]) {
  V3<T> mean = {0, 0, 0}, moment = {0, 0, 0};
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    mean = mean + v[c];
    moment = moment + cross(arm[c], v[c]);
  }
  mean = T(0.25) * mean;
  const V3<T> spin = symMul(inv, moment);
#pragma unroll
  for (int c = 0; c < 4; ++c) v[c] = v[c] - (mean + cross(spin, arm[c]));
}

// R K R^T p in the rotated frame: gh_c = R g_c, sigma = a tr(e) I + b e with
// e = sym(sum_b p_b gh_b^T), y_c = sigma gh_c  (a = lambda V, b = 2 mu V).
template <class T>
__device__ __forceinline__ void elasticProduct(const V3<T> gh[4], T a, T b, const V3<T> p[4], V3<T> y[4]) {
  M3<T> Q = zero3<T>();
#pragma unroll
  for (int c = 0; c < 4; ++c) addOuter(Q, p[c], gh[c]);
  const Sym<T> eps = symOf(Q);
  const T at = a * symTrace(eps);
  const Sym<T> sig = {at + b * eps.xx, at + b * eps.yy, at + b * eps.zz, b * eps.xy, b * eps.xz, b * eps.yz};
#pragma unroll
  for (int c = 0; c < 4; ++c) y[c] = symMul(sig, gh[c]);
}

template <class T>
__device__ __forceinline__ void dampingApply(const V3<T> arm[4], const Sym<T>& inv, const V3<T> gh[4], T a, T b,
                                             const V3<T> p[4], V3<T> y[4]) {
  V3<T> rel[4] = {p[0], p[1], p[2], p[3]};
  removeRigid(arm, inv, rel);
  elasticProduct(gh, a, b, rel, y);
  removeRigid(arm, inv, y);
}

// Inverse of the symmetric inertia tensor, or its pseudo-inverse keeping the
// eigenvalues above `floor` (factor.cc:183-272, 806-814); out of line, the
// degenerate branch is rare.
static __device__ __noinline__ Sym<double> inertiaInverse(Sym<double> I) {
  const double third = (I.xx + I.yy + I.zz) / 3.0;
  M3<double> m;
  m.m[0][0] = I.xx; m.m[1][1] = I.yy; m.m[2][2] = I.zz;
  m.m[0][1] = m.m[1][0] = I.xy;
  m.m[0][2] = m.m[2][0] = I.xz;
  m.m[1][2] = m.m[2][1] = I.yz;
  const double det = det3(m);
  if (det > 1.0e-6 * third * third * third) {
    const M3<double> c = cofactor(m);
    const double inv = 1.0 / det;
    return {c.m[0][0] * inv, c.m[1][1] * inv, c.m[2][2] * inv, c.m[0][1] * inv, c.m[0][2] * inv, c.m[1][2] * inv};
  }
  double a[3][3], v[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a[i][j] = m.m[i][j];
  jacobiEigen3(a, v);
  Sym<double> out = {0, 0, 0, 0, 0, 0};
  const double floor = 1.0e-6 * third;
  for (int k = 0; k < 3; ++k) {
    if (!(a[k][k] > floor)) continue;
    const double w = 1.0 / a[k][k];
    out.xx += w * v[0][k] * v[0][k];
    out.yy += w * v[1][k] * v[1][k];
    out.zz += w * v[2][k] * v[2][k];
    out.xy += w * v[0][k] * v[1][k];
    out.xz += w * v[0][k] * v[2][k];
    out.yz += w * v[1][k] * v[2][k];
  }
  return out;
}

// After the element pass of an assemble (corotated law): for every damped
// element, fit the rigid motion at the evaluated positions, keep the fit and
// the scaled coefficients for the matvec, subtract tau D(viscous velocity)
// from the corner forces and add the corner blocks of the damping operator to
// the diagonal records.  FP64 arithmetic; records stay in S.
template <class S>
__global__ void __launch_bounds__(TILE) kDamping(Sys<S> s, const Vec4<S>* base, const Vec4<S>* dir, uint32_t pass) {
  const uint32_t tile = blockIdx.x, b = s.elem_tile_body[tile];
  if (!bodyActive(s, b, pass)) return;
  const uint32_t e = tile * TILE + threadIdx.x;
  if (e >= s.body[b].elem_end) return;
  const double tau = double(s.dtau[e]);
  if (tau == 0.0) return;
  const BodyStepDev& st = s.step[b];
  const double reach = dir ? st.scale : 0.0;
  const uint4 t = __ldg(&s.tet[e]);
  const uint32_t nodes[4] = {t.x, t.y, t.z, t.w};
  // rigid fit at the evaluated corners (absolute positions)
  V3<double> arm[4], centre = {0, 0, 0};
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    V3<double> x = cvt<double>(xyz(ld4g(&s.rest4[nodes[c]]))) + cvt<double>(xyz(base[nodes[c]]));
    if (dir) x = x + reach * cvt<double>(xyz(dir[nodes[c]]));
    arm[c] = x;
    centre = centre + x;
  }
  centre = 0.25 * centre;
  Sym<double> inertia = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    arm[c] = arm[c] - centre;
    const V3<double>& q = arm[c];
    const double qq = dot(q, q);
    inertia.xx += qq - q.x * q.x;
    inertia.yy += qq - q.y * q.y;
    inertia.zz += qq - q.z * q.z;
    inertia.xy -= q.x * q.y;
    inertia.xz -= q.x * q.z;
    inertia.yz -= q.y * q.z;
  }
  const Sym<double> inv = inertiaInverse(inertia);
  // rotated gradients gh = R g from the committed rotation and Dm^-1
  M3<double> R;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) R.m[i][j] = double(s.op[size_t(3 * i + j) * s.Tp + e]);
  V3<double> g[4], gh[4];
  gradientsOf<S>(s.dm, s.Tp, e, g);
#pragma unroll
  for (int c = 0; c < 4; ++c) gh[c] = mul(R, g[c]);
  const MatDev m = s.mat[s.lane[e]];
  const double youngs = s.eyoung ? s.eyoung[e] : m.youngs;
  const double vol = s.vold[e];
  const double a = youngs * m.lam_unit * vol, bb = 2.0 * youngs * m.mu_unit * vol;
  const double dscale = (1.0 - st.alpha_f) * st.gamma * st.inner;  // Damping::scale
  // the fit and the scaled coefficients for the matvec
  const double keep[20] = {arm[0].x, arm[0].y, arm[0].z, arm[1].x, arm[1].y, arm[1].z, arm[2].x, arm[2].y,
                           arm[2].z, arm[3].x, arm[3].y, arm[3].z, inv.xx,   inv.yy,   inv.zz,   inv.xy,
                           inv.xz,   inv.yz,   dscale * tau * a, dscale * tau * bb};
#pragma unroll
  for (int k = 0; k < 20; ++k) s.dfit[size_t(k) * s.Tp + e] = S(keep[k]);
  // viscous force of the lagged velocity (anchored nodes: zero)
  const double lag = (1.0 - st.alpha_f) * st.inner;
  V3<double> vv[4], dv[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const uint32_t n = nodes[c];
    if (s.anch[n]) {
      vv[c] = {0, 0, 0};
      continue;
    }
    // a floating body's viscous velocity is its frame velocity (solver.cc:3757-3759)
    vv[c] = cvt<double>(xyz(st.floating ? s.relv[n] : s.v[n])) + (lag * (1.0 - st.gamma)) * cvt<double>(xyz(s.carried[n]));
    if (dir) vv[c] = vv[c] + (lag * st.gamma) * cvt<double>(xyz(dir[n]));
  }
  dampingApply(arm, inv, gh, a, bb, vv, dv);
  // diagonal corner blocks of D, scaled like the element blocks (the node
  // gather multiplies the records by h_eff^2)
  const double wdiag = dscale * tau / st.scale;
#pragma unroll 1
  for (int c = 0; c < 4; ++c) {
    M3<double> blk;
#pragma unroll 1
    for (int axis = 0; axis < 3; ++axis) {
      V3<double> unit[4] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, col[4];
      if (axis == 0) unit[c].x = 1.0;
      else if (axis == 1) unit[c].y = 1.0;
      else unit[c].z = 1.0;
      dampingApply(arm, inv, gh, a, bb, unit, col);
      blk.m[0][axis] = col[c].x;
      blk.m[1][axis] = col[c].y;
      blk.m[2][axis] = col[c].z;
    }
    const size_t at = size_t(c) * s.Tp + e;
    const Vec4<S> f = s.fe[at], d = s.de[at];
    s.fe[at] = Vec4<S>{S(double(f.x) - tau * dv[c].x), S(double(f.y) - tau * dv[c].y),
                       S(double(f.z) - tau * dv[c].z), S(double(f.w) + wdiag * blk.m[0][0])};
    s.de[at] = Vec4<S>{S(double(d.x) + wdiag * blk.m[1][1]), S(double(d.y) + wdiag * blk.m[2][2]),
                       S(double(d.z) + wdiag * 0.5 * (blk.m[0][1] + blk.m[1][0])),
                       S(double(d.w) + wdiag * 0.5 * (blk.m[0][2] + blk.m[2][0]))};
    s.de2[at] = S(double(s.de2[at]) + wdiag * 0.5 * (blk.m[1][2] + blk.m[2][1]));
  }
}

// Matvec share of damping for one element: y += (1 - alpha_f) gamma h tau D(p),
// in S, from the fit kept by kDamping and the rotated gradients gh.  Only the
// DAMP instantiations of the PCG kernels (systems with stiffness damping)
// contain it.
template <class S>
__device__ __forceinline__ void dampingProduct(const Sys<S>& s, uint32_t e, const V3<S> gh[4], const V3<S> p[4],
                                               V3<S> y[4]) {
  if (s.dtau[e] == S(0)) return;
  S k[20];
#pragma unroll
  for (int q = 0; q < 20; ++q) k[q] = s.dfit[size_t(q) * s.Tp + e];
  const V3<S> arm[4] = {{k[0], k[1], k[2]}, {k[3], k[4], k[5]}, {k[6], k[7], k[8]}, {k[9], k[10], k[11]}};
  const Sym<S> inv = {k[12], k[13], k[14], k[15], k[16], k[17]};
  V3<S> d[4];
  dampingApply(arm, inv, gh, k[18], k[19], p, d);
#pragma unroll
  for (int c = 0; c < 4; ++c) y[c] = y[c] + d[c];
}

// ------------------------------------------------- state transfer ----
// A body's committed rotations and plastic points between the caller's
// per-tet layout (DeformableState, mesh.h:56-62: the rotation's 9 entries
// row-major; the plastic strain's 9 entries row-major, then the equivalent
// strain) and the element planes (op; plast as (exx, eyy, ezz, exy),
// (exz, eyz, equivalent, -), off-diagonals averaged in FP64).  Tet t of the
// body is element e0 + t; null arrays are skipped.
template <class S, class H>
__global__ void __launch_bounds__(TILE) kElemStateIn(Sys<S> s, uint32_t e0, uint32_t T, const H* rot,
                                                     const H* plastic) {
  const uint32_t t = blockIdx.x * TILE + threadIdx.x;
  if (t >= T) return;
  const size_t e = size_t(e0) + t;
  if (rot) {
#pragma unroll
    for (int k = 0; k < 9; ++k) s.op[size_t(k) * s.Tp + e] = S(rot[9 * size_t(t) + k]);
  }
  if (plastic && s.hk) {  // finite-strain flow: P row-major, hardening variable
#pragma unroll
    for (int k = 0; k < 10; ++k) s.hk[size_t(k) * s.Tp + e] = double(plastic[10 * size_t(t) + k]);
  } else if (plastic) {
    const H* q = plastic + 10 * size_t(t);
    s.plast[e] = Vec4<S>{S(q[0]), S(q[4]), S(q[8]), S(0.5 * (double(q[1]) + double(q[3])))};
    s.plast[size_t(s.Tp) + e] = Vec4<S>{S(0.5 * (double(q[2]) + double(q[6]))),
                                        S(0.5 * (double(q[5]) + double(q[7]))), S(q[9]), S(0)};
  }
}

template <class S, class H>
__global__ void __launch_bounds__(TILE) kElemStateOut(Sys<S> s, uint32_t e0, uint32_t T, H* rot, H* plastic) {
  const uint32_t t = blockIdx.x * TILE + threadIdx.x;
  if (t >= T) return;
  const size_t e = size_t(e0) + t;
  if (rot) {
#pragma unroll
    for (int k = 0; k < 9; ++k) rot[9 * size_t(t) + k] = H(s.op[size_t(k) * s.Tp + e]);
  }
  if (plastic && s.hk) {
#pragma unroll
    for (int k = 0; k < 10; ++k) plastic[10 * size_t(t) + k] = H(s.hk[size_t(k) * s.Tp + e]);
  } else if (plastic) {
    H* q = plastic + 10 * size_t(t);
    const Vec4<S> a0 = s.plast[e], a1 = s.plast[size_t(s.Tp) + e];
    q[0] = H(a0.x); q[1] = H(a0.w); q[2] = H(a1.x);
    q[3] = H(a0.w); q[4] = H(a0.y); q[5] = H(a1.y);
    q[6] = H(a1.x); q[7] = H(a1.y); q[8] = H(a0.z);
    q[9] = H(a1.z);
  }
}

// -------------------------------------------- finite-strain plastic flow ----
__device__ inline M3<double> inverse3(const M3<double>& a) {
  const M3<double> c = cofactor(a);
  const double inv = 1.0 / det3(a);
  M3<double> r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r.m[i][j] = c.m[j][i] * inv;
  return r;
}

// flowLattice (plasticflow.cc:184-247) once per step after the solve
// (strainstep.cc:822-825), one point per tet.  The elastic map F P returns
// with the yield stress blended toward the trial stress, (start + r q) /
// (1 + r), r = H / (3 mu).  A crushable lane (finite crush stress, crush
// limit < 1) squeezed below J = exp(-crushStress / K) compacts by
// min(-crush - log J, room), room = -log(det P crushLimit).  P becomes
// F^-1 (grow Fe,returned); a plastic stretch Fp further than the lane's cap
// from I (Frobenius) is pulled back to that distance at the same volume.  P
// is written when it moves by more than 1e-12 (one-norm) and the hardening
// variable grows by the returned strain.  Flowed tets are counted into the
// body's yielding counter.
template <class S>
__global__ void __launch_bounds__(TILE) kHenckyFlow(Sys<S> s) {
  const uint32_t tile = blockIdx.x, b = s.elem_tile_body[tile];
  const uint32_t e = tile * TILE + threadIdx.x;
  bool flowed = false;
  if (e < s.body[b].elem_end) {
    const uint32_t lane = s.lane[e];
    const MatDev m = s.mat[lane];
    if (m.yields) {
      const uint4 t = __ldg(&s.tet[e]);
      const uint32_t nodes[4] = {t.x, t.y, t.z, t.w};
      V3<double> g[4];
      gradientsOf<S>(s.dm, s.Tp, e, g);
      M3<double> F = eye3<double>();
#pragma unroll
      for (int c = 0; c < 4; ++c) addOuter(F, cvt<double>(xyz(s.u[nodes[c]])), g[c]);
      if (det3(F) > 0.0) {
        M3<double> P;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) P.m[i][j] = s.hk[size_t(3 * i + j) * s.Tp + e];
        const double hardening = s.hk[size_t(9) * s.Tp + e];
        const double youngs = s.eyoung ? s.eyoung[e] : m.youngs;
        const double mu = youngs * m.mu_unit, bulk = youngs * m.lam_unit + 2.0 * mu / 3.0;
        const double hard = m.hardening;
        const double crushStress = s.flim[3 * lane], crushLimit = s.flim[3 * lane + 1], cap = s.flim[3 * lane + 2];
        const bool crushable = isfinite(crushStress) && crushLimit < 1.0;
        const double crush = crushStress / bulk;
        const M3<double> fe = mul(F, P);
        const double start = m.yield + hard * hardening;
        const double room = crushable ? -log(det3(P) * crushLimit) : 0.0;
        const bool squeezed = crushable && room > 0.0 && det3(fe) < exp(-crush);
        M3<double> back = fe;
        double strain = 0.0, trial = 0.0;
        bool mapped = false;
        if (henckyReturn(fe, mu, start, back, strain, trial)) {
          const double ratio = hard / (3.0 * mu);
          const double yieldNow = (start + ratio * trial) / (1.0 + ratio);
          mapped = henckyReturn(fe, mu, yieldNow, back, strain, trial);
        }
        const M3<double> after = mapped ? back : fe;
        const double volume = det3(after);
        const double compaction = squeezed && volume > 0.0 ? fmin(-crush - log(volume), room) : 0.0;
        if (mapped || compaction > 0.0) {
          const double grow = compaction > 0.0 ? exp(compaction / 3.0) : 1.0;
          M3<double> grown = after;
#pragma unroll
          for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) grown.m[i][j] *= grow;
          M3<double> next = mul(inverse3(F), grown);
          const double kept = det3(next);
          bool keep = true;
          if (isfinite(cap) && kept > 0.0) {
            M3<double> stretch = inverse3(next);
            stretch.m[0][0] -= 1.0;
            stretch.m[1][1] -= 1.0;
            stretch.m[2][2] -= 1.0;
            const double size = sqrt(contract(stretch, stretch));
            if (size > cap) {
              M3<double> capped;
#pragma unroll
              for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) capped.m[i][j] = (i == j ? 1.0 : 0.0) + (cap / size) * stretch.m[i][j];
              const double cappedVolume = det3(capped);
              keep = cappedVolume > 1.0e-6;
              if (keep) {
                const double scale = cbrt(kept * cappedVolume);
                next = inverse3(capped);
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                  for (int j = 0; j < 3; ++j) next.m[i][j] *= scale;
              }
            }
          }
          double moved = 0.0;
#pragma unroll
          for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) moved += fabs(next.m[i][j] - P.m[i][j]);
          if (keep && moved > 1.0e-12) {
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
              for (int j = 0; j < 3; ++j) s.hk[size_t(3 * i + j) * s.Tp + e] = next.m[i][j];
            s.hk[size_t(9) * s.Tp + e] = hardening + (mapped ? strain : 0.0);
            flowed = true;
          }
        }
      }
    }
  }
  const int n = __syncthreads_count(flowed);
  if (threadIdx.x == 0 && n) {
    atomicAdd(&s.yielding[b], uint32_t(n));
    atomicOr(&s.acc[b].grew, 1u);
  }
}

// ---------------------------------------------------------------- PCG ----

// h_eff^2 (R K R^T p)_e for one tet: applyStiffness (material.cc:267-288) with
// the elastic blocks of tetStiffness (material.cc:209-234) or the consistent
// tangent of tetPointTrial (material.cc:1033-1054), in the rotated frame where
// gh = R g:  Q = sum_b p_b gh_b^T, e = sym(Q), sigma = a tr(e) I + b e -
// c (nh : e) nh, y_a = sigma gh_a.  LAW 1: the exact SNH tangent dP(dF) g_a
// with dF = sum_b p_b g_b^T.  (a, b, c) carry h_eff^2 V.  Arithmetic in S.
// The per-element matvec operator: rotated gradients gh_1..3 (g_0 = -sum),
// coefficients k, and the flow normal (corotated tangent) or F (SNH).
template <class S> struct ElementOperator {
  V3<S> g[4];
  Vec4<S> k;
  Sym<S> n;
  M3<S> F;
};

// The operator from the record's pieces q0..q2 (the flow normal pair for the
// corotated tangent; F from the op planes for SNH).
template <class S>
__device__ __forceinline__ void unpackOperator(ElementOperator<S>& o, Vec4<S> q0, Vec4<S> q1, Vec4<S> q2) {
  o.g[1] = {q0.x, q0.y, q0.z};
  o.g[2] = {q0.w, q1.x, q1.y};
  o.g[3] = {q1.z, q1.w, q2.x};
  o.g[0] = -(o.g[1] + o.g[2] + o.g[3]);
  o.k = Vec4<S>{q2.y, q2.z, q2.w, S(0)};
}

template <class S, int LAW, bool TANGENT>
__device__ __forceinline__ ElementOperator<S> loadOperator(const Sys<S>& s, uint32_t e) {
  ElementOperator<S> o;
  const OpRec<S>* rec = s.orec + e;
  unpackOperator(o, ld4g(&rec->q[0]), ld4g(&rec->q[1]), ld4g(&rec->q[2]));
  if (LAW == 0 && TANGENT) {
    const Vec4<S> n0 = ld4g(&s.onorm[2 * size_t(e)]), n1 = ld4g(&s.onorm[2 * size_t(e) + 1]);
    o.n = {n0.x, n0.y, n0.z, n0.w, n1.x, n1.y};
  }
  if (LAW == 1) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) o.F.m[i][j] = __ldg(s.op + size_t(3 * i + j) * s.Tp + e);
  }
  return o;
}

// ---- shared-memory stage of one tile's operators, filled by cp.async ----
// Layout: the tile's records [TILE] OpRec<S>, then for the corotated tangent
// its flow normal pairs [TILE][2] Vec4<S>, then for SNH op [9][TILE] S.
// Records and pairs are contiguous both in global and in shared memory, so
// each warp copies its 32 elements' span in 16-byte chunks with consecutive
// lanes on consecutive chunks (a per-thread copy of its own 48-byte record
// would fetch every 32-byte sector twice).  A thread then reads entries that
// other lanes copied: the caller orders the copies with cp.async.wait_group
// followed by a block barrier.
template <class S, int LAW, bool TANGENT> __host__ __device__ constexpr size_t stageBytes() {
  return sizeof(OpRec<S>) * TILE + (LAW == 0 && TANGENT ? sizeof(Vec4<S>) * 2 * TILE : 0) +
         (LAW == 1 ? sizeof(S) * 9 * TILE : 0);
}

// e: this thread's element (tile * TILE + threadIdx.x, below Tp).
template <class S, int LAW, bool TANGENT>
__device__ __forceinline__ void stageOperator(const Sys<S>& s, uint32_t e, unsigned char* stage) {
  const uint32_t t = threadIdx.x, lane = t & 31u, first = t & ~31u;  // the warp's first element in the tile
  {
    constexpr uint32_t CHUNKS = uint32_t(sizeof(OpRec<S>)) * 32u / 16u;
    const unsigned char* src = reinterpret_cast<const unsigned char*>(s.orec + (e - lane));
    unsigned char* dst = stage + size_t(first) * sizeof(OpRec<S>);
#pragma unroll
    for (uint32_t c = lane; c < CHUNKS; c += 32u) cpAsync<16>(dst + 16 * c, src + 16 * c);
  }
  if (LAW == 0 && TANGENT) {
    constexpr uint32_t CHUNKS = uint32_t(sizeof(Vec4<S>)) * 2u * 32u / 16u;
    const unsigned char* src = reinterpret_cast<const unsigned char*>(s.onorm + 2 * size_t(e - lane));
    unsigned char* dst = stage + sizeof(OpRec<S>) * TILE + size_t(first) * 2 * sizeof(Vec4<S>);
#pragma unroll
    for (uint32_t c = lane; c < CHUNKS; c += 32u) cpAsync<16>(dst + 16 * c, src + 16 * c);
  }
  if (LAW == 1) {
    S* op = reinterpret_cast<S*>(stage + sizeof(OpRec<S>) * TILE);
#pragma unroll
    for (int k = 0; k < 9; ++k) cpAsync<sizeof(S)>(op + k * TILE + t, s.op + size_t(k) * s.Tp + e);
  }
}

template <class S, int LAW, bool TANGENT>
__device__ __forceinline__ ElementOperator<S> stagedOperator(const unsigned char* stage) {
  const uint32_t t = threadIdx.x;
  const OpRec<S>& rec = reinterpret_cast<const OpRec<S>*>(stage)[t];
  ElementOperator<S> o;
  unpackOperator(o, rec.q[0], rec.q[1], rec.q[2]);
  if (LAW == 0 && TANGENT) {
    const Vec4<S>* nq = reinterpret_cast<const Vec4<S>*>(stage + sizeof(OpRec<S>) * TILE) + 2 * size_t(t);
    o.n = {nq[0].x, nq[0].y, nq[0].z, nq[0].w, nq[1].x, nq[1].y};
  }
  if (LAW == 1) {
    const S* op = reinterpret_cast<const S*>(stage + sizeof(OpRec<S>) * TILE);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) o.F.m[i][j] = op[(3 * i + j) * TILE + t];
  }
  return o;
}

template <class S, int LAW, bool TANGENT>
__device__ __forceinline__ void applyOperator(const ElementOperator<S>& o, const V3<S> p[4], V3<S> y[4]) {
  const V3<S>* g = o.g;
  const Vec4<S> k = o.k;
  M3<S> Q = zero3<S>();
#pragma unroll
  for (int c = 1; c < 4; ++c) addOuter(Q, p[c] - p[0], g[c]);  // sum_c g_c = 0
  if (LAW == 0) {
    const Sym<S> eps = symOf(Q);
    const S tr = symTrace(eps);
    const S at = k.x * tr;
    Sym<S> sig = {at + k.y * eps.xx, at + k.y * eps.yy, at + k.y * eps.zz, k.y * eps.xy, k.y * eps.xz, k.y * eps.yz};
    if (TANGENT) {
      const Sym<S>& n = o.n;
      const S ne = k.z * symContract(n, eps);
      sig.xx -= ne * n.xx;
      sig.yy -= ne * n.yy;
      sig.zz -= ne * n.zz;
      sig.xy -= ne * n.xy;
      sig.xz -= ne * n.xz;
      sig.yz -= ne * n.yz;
    }
#pragma unroll
    for (int c = 1; c < 4; ++c) y[c] = symMul(sig, g[c]);
  } else {
    const M3<S>& F = o.F;
    const M3<S> C = cofactor(F);
    const S kk = k.z * contract(C, Q);
    // column j of cof F is F_{j+1} x F_{j+2}; its differential along Q
    M3<S> dP;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
      const V3<S> f1 = {F.m[0][j1], F.m[1][j1], F.m[2][j1]}, f2 = {F.m[0][j2], F.m[1][j2], F.m[2][j2]};
      const V3<S> d1 = {Q.m[0][j1], Q.m[1][j1], Q.m[2][j1]}, d2 = {Q.m[0][j2], Q.m[1][j2], Q.m[2][j2]};
      const V3<S> dcof = cross(d1, f2) + cross(f1, d2);
      dP.m[0][j] = k.x * Q.m[0][j] + k.y * dcof.x + kk * C.m[0][j];
      dP.m[1][j] = k.x * Q.m[1][j] + k.y * dcof.y + kk * C.m[1][j];
      dP.m[2][j] = k.x * Q.m[2][j] + k.y * dcof.z + kk * C.m[2][j];
    }
#pragma unroll
    for (int c = 1; c < 4; ++c) y[c] = mul(dP, g[c]);
  }
  y[0] = -(y[1] + y[2] + y[3]);
}

template <class S, int LAW, bool TANGENT, bool DAMP = false>
__device__ __forceinline__ void elementApply(const Sys<S>& s, uint32_t e, const V3<S> p[4], V3<S> y[4]) {
  const ElementOperator<S> o = loadOperator<S, LAW, TANGENT>(s, e);
  applyOperator<S, LAW, TANGENT>(o, p, y);
  if (DAMP && LAW == 0) dampingProduct(s, e, o.g, p, y);
}

// Reads a body's PCG scalars from L2 (they are written by other blocks).
__device__ __forceinline__ CgBodyDev loadCg(const CgBodyDev* p) {
  CgBodyDev c;
  c.squared = __ldcg(&p->squared);
  c.target = __ldcg(&p->target);
  c.floor = __ldcg(&p->floor);
  c.length = __ldcg(&p->length);
  c.stride = __ldcg(&p->stride);
  c.blend = __ldcg(&p->blend);
  c.start_res = __ldcg(&p->start_res);
  c.rel_res = __ldcg(&p->rel_res);
  c.taken = __ldcg(&p->taken);
  c.done = __ldcg(&p->done);
  c.pad0 = c.pad1 = 0;
  return c;
}

template <class S> __device__ __forceinline__ V3<S> fmaV(S a, V3<S> x, V3<S> y) {
  return {fma(a, x.x, y.x), fma(a, x.y, y.y), fma(a, x.z, y.z)};
}

// Persistent PCG over every body of the system (conjugateGradient,
// solver.cc:1904-2089, block-Jacobi branch).  One cooperative launch runs all
// iterations; each body keeps its own scalars and stops on its own test, and
// the launch ends when no body iterates.  Three grid barriers per iteration:
//   A (element tiles) y_e = scale R K R^T p_e with p = z + blend p_prev formed on the fly
//   B (node tiles)    p = z + blend p_prev; Ap = inertia m p + sum y_e; p.Ap
//   C (node tiles)    x += stride p; r -= stride Ap; z = P r; r.z, r.r
template <class S, int LAW>
__global__ void __launch_bounds__(TILE, 2)
    kPcg(Sys<S> s, Vec4<S>* X, uint32_t pass, uint32_t x0zero, uint32_t tangent) {
  const uint32_t G = gridDim.x;
  const S zero = S(0);
  // ---- init: r = right - A x (anchored rows 0), z = P r, p_prev = 0
  if (!x0zero) {
    for (uint32_t tile = blockIdx.x; tile < s.elem_tiles; tile += G) {
      const uint32_t b = s.elem_tile_body[tile];
      if (!bodyActive(s, b, pass)) continue;
      const uint32_t e = tile * TILE + threadIdx.x;
      if (e >= s.body[b].elem_end) continue;
      const uint4 t = __ldg(&s.tet[e]);
      const uint32_t nodes[4] = {t.x, t.y, t.z, t.w};
      V3<S> pe[4], y[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) pe[c] = xyz(ld4cg(&X[nodes[c]]));
      if (tangent) elementApply<S, LAW, true>(s, e, pe, y);
      else elementApply<S, LAW, false>(s, e, pe, y);
#pragma unroll
      for (int c = 0; c < 4; ++c) s.ye[4 * e + c] = pack(y[c]);
    }
    if (!gridBarrier(s.sync)) return;
  }
  for (uint32_t tile = blockIdx.x; tile < s.node_tiles; tile += G) {
    const uint32_t b = s.node_tile_body[tile];
    if (!bodyActive(s, b, pass)) continue;
    const uint32_t n = tile * TILE + threadIdx.x;
    double sums[3] = {0.0, 0.0, 0.0};
    if (n < s.body[b].node_end) {
      const Vec4<S> rhs = s.right[n];
      V3<S> r = {zero, zero, zero};
      if (!s.anch[n]) {
        V3<double> ax = {0, 0, 0};
        if (!x0zero) {
          const double im = s.step[b].inertia * double(ld4g(&s.rest4[n]).w);
          ax = im * cvt<double>(xyz(ld4cg(&X[n])));
          for (uint32_t k = s.start[n]; k < s.start[n + 1]; ++k) ax = ax + cvt<double>(xyz(ld4cg(&s.ye[__ldg(&s.entry[k])])));
        }
        r = cvt<S>(cvt<double>(xyz(rhs)) - ax);
      }
      const Vec4<S> q0 = s.pre0[n], q1 = s.pre1[n];
      const Sym<S> P = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y};
      const V3<S> z = symMul(P, r);
      s.r[n] = pack(r);
      s.z[n] = pack(z);
      s.p[n] = Vec4<S>{zero, zero, zero, zero};
      if (x0zero) X[n] = Vec4<S>{zero, zero, zero, zero};
      sums[0] = dot(cvt<double>(r), cvt<double>(z));
      sums[1] = dot(cvt<double>(r), cvt<double>(r));
      sums[2] = dot(cvt<double>(xyz(rhs)), cvt<double>(xyz(rhs)));
    }
    blockSum<3>(sums);
    if (threadIdx.x == 0) {
      s.part[size_t(tile) * 4 + 0] = sums[0];
      s.part[size_t(tile) * 4 + 1] = sums[1];
      s.part[size_t(tile) * 4 + 2] = sums[2];
    }
    const BodyDev bd = s.body[b];
    if (lastTileOfBody(&s.counter[b], bd.node_tile_end - bd.node_tile_begin)) {
      double tot[3];
      sumTiles<3>(s.part, bd.node_tile_begin, bd.node_tile_end, tot);
      if (threadIdx.x == 0) {
        CgBodyDev c;
        const double reference = sqrt(tot[2]);
        c.floor = fmax(reference, 1.1754943508222875e-38);  // std::numeric_limits<float>::min()
        c.target = s.step[b].tolerance * c.floor;
        c.squared = tot[0];
        c.length = tot[1];
        c.start_res = sqrt(tot[1]) / c.floor;
        c.rel_res = c.start_res;
        c.blend = 0.0;
        c.stride = 0.0;
        c.taken = 0;
        c.done = (s.step[b].limit == 0u || sqrt(c.length) <= c.target) ? 1u : 0u;
        c.pad0 = c.pad1 = 0;
        s.cg[b] = c;
        __threadfence();
        if (c.done) atomicSub(&s.sync->active, 1);
      }
    }
  }
  if (!gridBarrier(s.sync)) return;
  for (;;) {
    if (*(volatile int*)&s.sync->active <= 0) break;  // uniform: no block decrements between here and barrier A
    // ---- A
    for (uint32_t tile = blockIdx.x; tile < s.elem_tiles; tile += G) {
      const uint32_t b = s.elem_tile_body[tile];
      if (!bodyActive(s, b, pass) || __ldcg(&s.cg[b].done)) continue;
      const uint32_t e = tile * TILE + threadIdx.x;
      if (e >= s.body[b].elem_end) continue;
      const S blend = S(__ldcg(&s.cg[b].blend));
      const uint4 t = __ldg(&s.tet[e]);
      const uint32_t nodes[4] = {t.x, t.y, t.z, t.w};
      V3<S> pe[4], y[4];
#pragma unroll
      for (int c = 0; c < 4; ++c)
        pe[c] = fmaV(blend, xyz(ld4cg(&s.p[nodes[c]])), xyz(ld4cg(&s.z[nodes[c]])));
      if (tangent) elementApply<S, LAW, true>(s, e, pe, y);
      else elementApply<S, LAW, false>(s, e, pe, y);
#pragma unroll
      for (int c = 0; c < 4; ++c) s.ye[4 * e + c] = pack(y[c]);
    }
    if (!gridBarrier(s.sync)) return;
    // ---- B
    for (uint32_t tile = blockIdx.x; tile < s.node_tiles; tile += G) {
      const uint32_t b = s.node_tile_body[tile];
      if (!bodyActive(s, b, pass) || __ldcg(&s.cg[b].done)) continue;
      const uint32_t n = tile * TILE + threadIdx.x;
      double sums[1] = {0.0};
      if (n < s.body[b].node_end) {
        const S blend = S(__ldcg(&s.cg[b].blend));
        const V3<S> pn = fmaV(blend, xyz(ld4cg(&s.p[n])), xyz(ld4cg(&s.z[n])));
        s.p[n] = pack(pn);
        V3<S> apn = {zero, zero, zero};
        if (!s.anch[n]) {
          V3<double> acc = (s.step[b].inertia * double(ld4g(&s.rest4[n]).w)) * cvt<double>(pn);
          for (uint32_t k = s.start[n]; k < s.start[n + 1]; ++k)
            acc = acc + cvt<double>(xyz(ld4cg(&s.ye[__ldg(&s.entry[k])])));
          apn = cvt<S>(acc);
        }
        s.ap[n] = pack(apn);
        sums[0] = dot(cvt<double>(pn), cvt<double>(apn));
      }
      blockSum<1>(sums);
      if (threadIdx.x == 0) s.part[size_t(tile) * 4 + 3] = sums[0];
      const BodyDev bd = s.body[b];
      if (lastTileOfBody(&s.counter[b], bd.node_tile_end - bd.node_tile_begin)) {
        double tot[1];
        double* base = s.part + 3;
        sumTiles<1>(base, bd.node_tile_begin, bd.node_tile_end, tot);
        if (threadIdx.x == 0) {
          const double curvature = tot[0];
          const double squared = __ldcg(&s.cg[b].squared);
          if (!(curvature > 0.0) || !(squared > 0.0)) {
            s.cg[b].done = 1u;
            __threadfence();
            atomicSub(&s.sync->active, 1);
          } else {
            s.cg[b].stride = squared / curvature;
            __threadfence();
          }
        }
      }
    }
    // No exit test here: phase C finalizers may already be decrementing the
    // active count in other blocks.  The count is read only at the loop top,
    // where every writer is ordered behind the previous barrier.
    if (!gridBarrier(s.sync)) return;
    // ---- C
    for (uint32_t tile = blockIdx.x; tile < s.node_tiles; tile += G) {
      const uint32_t b = s.node_tile_body[tile];
      if (!bodyActive(s, b, pass) || __ldcg(&s.cg[b].done)) continue;
      const uint32_t n = tile * TILE + threadIdx.x;
      double sums[2] = {0.0, 0.0};
      if (n < s.body[b].node_end) {
        const S stride = S(__ldcg(&s.cg[b].stride));
        const V3<S> pn = xyz(ld4cg(&s.p[n]));
        const V3<S> x = fmaV(stride, pn, xyz(ld4cg(&X[n])));
        const V3<S> r = fmaV(-stride, xyz(ld4cg(&s.ap[n])), xyz(ld4cg(&s.r[n])));
        const Vec4<S> q0 = s.pre0[n], q1 = s.pre1[n];
        const Sym<S> P = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y};
        const V3<S> z = symMul(P, r);
        X[n] = pack(x);
        s.r[n] = pack(r);
        s.z[n] = pack(z);
        sums[0] = dot(cvt<double>(r), cvt<double>(z));
        sums[1] = dot(cvt<double>(r), cvt<double>(r));
      }
      blockSum<2>(sums);
      if (threadIdx.x == 0) {
        s.part[size_t(tile) * 4 + 0] = sums[0];
        s.part[size_t(tile) * 4 + 1] = sums[1];
      }
      const BodyDev bd = s.body[b];
      if (lastTileOfBody(&s.counter[b], bd.node_tile_end - bd.node_tile_begin)) {
        double tot[2];
        sumTiles<2>(s.part, bd.node_tile_begin, bd.node_tile_end, tot);
        if (threadIdx.x == 0) {
          CgBodyDev c = loadCg(&s.cg[b]);
          c.blend = tot[0] / c.squared;
          c.squared = tot[0];
          c.length = tot[1];
          c.taken += 1u;
          c.done = (sqrt(c.length) <= c.target || c.taken >= s.step[b].limit) ? 1u : 0u;
          s.cg[b] = c;
          __threadfence();
          if (c.done) atomicSub(&s.sync->active, 1);
        }
      }
    }
    if (!gridBarrier(s.sync)) return;
  }
  // ---- per-body results (block 0)
  if (blockIdx.x == 0) {
    for (uint32_t b = threadIdx.x; b < s.bodies; b += TILE) {
      if (!bodyActive(s, b, pass)) continue;
      CgBodyDev c = loadCg(&s.cg[b]);
      const double residual = sqrt(c.length);
      c.rel_res = residual / c.floor;
      s.cg[b].rel_res = c.rel_res;
      CgReportDev rep = s.cgrep[b];
      rep.iterations += c.taken;
      rep.capped += (c.taken == s.step[b].limit && residual > c.target) ? 1u : 0u;
      rep.applications += c.taken + (x0zero ? 0u : 1u);
      rep.solves += 1u;
      rep.tangent_iterations += tangent ? c.taken : 0u;
      rep.worst_rel = fmax(rep.worst_rel, c.rel_res);
      if (rep.pass_solves == 0u) rep.pass_start = c.start_res;
      rep.pass_end = c.rel_res;
      rep.pass_iterations += c.taken;
      rep.pass_solves += 1u;
      s.cgrep[b] = rep;
    }
  }
}

// ------------------------------------------------ single-body fast PCG ----

// Release add without a returned value: the arriving block starts polling
// without waiting for the atomic's reply (its own later load of the counter
// sees the add, which precedes it in program order on the same address).
__device__ __forceinline__ void redAddRelease(unsigned int* p, unsigned int v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned int ldAcquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Counting grid barrier: barrier k of a launch completes when the arrival
// counter (zeroed before the launch) reaches gridDim.x * k.  Release on
// arrival, acquire while polling; the wait is bounded by TL_BARRIER_LIMIT_NS,
// after which the block records TL_ERR_TIMEOUT and every block leaves.
__device__ __forceinline__ bool countBarrier(GridSyncDev* sync, unsigned int& k) {
  __shared__ int ok;
  ++k;
  __syncthreads();
  if (threadIdx.x == 0) {
    int good = 1;
    const unsigned int goal = gridDim.x * k;
    redAddRelease(&sync->arrive, 1u);
    if (ldAcquire(&sync->arrive) < goal) {
      const unsigned long long t0 = globalTimer();
      unsigned int polls = 0;
      while (ldAcquire(&sync->arrive) < goal) {
        if ((++polls & 255u) == 0u) {
          if (*(volatile int*)&sync->error != 0) {
            good = 0;
            break;
          }
          if (globalTimer() - t0 > TL_BARRIER_LIMIT_NS) {
            atomicExch(&sync->error, 5);  // TL_ERR_TIMEOUT
            good = 0;
            break;
          }
        }
      }
    }
    ok = good;
  }
  __syncthreads();
  return ok != 0;
}

// Sums of fields [0, N) of every block's partials (field k of block b at
// part[k G + b]) in one pass, the same in every block: all threads load at
// once (thread t adds blocks t, t + TILE, ...), then a fixed shuffle tree per
// warp and the warps in order, so a grid barrier is followed by one L2 round
// trip instead of one per block stride.
template <int N>
__device__ __forceinline__ void sumBlocksAll(const double* part, double (&out)[N]) {
  __shared__ double red[N][TILE / 32];
  const unsigned G = gridDim.x;
  double v[N];
#pragma unroll
  for (int k = 0; k < N; ++k) v[k] = 0.0;
  for (unsigned b = threadIdx.x; b < G; b += TILE)
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] += __ldcg(part + size_t(k) * G + b);
#pragma unroll
  for (int k = 0; k < N; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int k = 0; k < N; ++k) red[k][threadIdx.x >> 5] = v[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < N; ++k) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < TILE / 32; ++w) t += red[k][w];
    out[k] = t;
  }
  __syncthreads();
}

// The first `fields` G partials of part (field k of block b at part[k G + b]),
// requested into shared memory by cp.async in 16-byte pieces through L2 and
// committed as one group; the caller waits for it (cp.async.wait_group 0),
// then a block barrier, before sumStagedBlocks reads them.  part is 16-byte
// aligned and holds at least fields G + 1 values.
__device__ __forceinline__ void requestBlockPartials(const double* part, double* stage, unsigned fields) {
  const unsigned pieces = (fields * gridDim.x + 1u) / 2u;
  for (unsigned i = threadIdx.x; i < pieces; i += TILE) cpAsync<16>(stage + 2 * i, part + 2 * i);
  cpAsyncCommit();
}
// sumBlocksAll on partials staged by requestBlockPartials: the same order of
// additions, so the same sums.
template <int N>
__device__ __forceinline__ void sumStagedBlocks(const double* stage, double (&out)[N]) {
  __shared__ double red[N][TILE / 32];
  const unsigned G = gridDim.x;
  double v[N];
#pragma unroll
  for (int k = 0; k < N; ++k) v[k] = 0.0;
  for (unsigned b = threadIdx.x; b < G; b += TILE)
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] += stage[size_t(k) * G + b];
#pragma unroll
  for (int k = 0; k < N; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int k = 0; k < N; ++k) red[k][threadIdx.x >> 5] = v[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < N; ++k) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < TILE / 32; ++w) t += red[k][w];
    out[k] = t;
  }
  __syncthreads();
}

// One element tile of the matvec: y_e = h_eff^2 (R K R^T p)_e for its 256
// elements, then the tile-local sums of y_e per touched node, in ascending
// element order, written to the tile's slots.  The tile's distinct nodes are
// staged once in shared memory (p = z + blend p_prev formed once per node, or
// X for the initial residual), elements read their corners from there by
// local index, and the tile's local CSR is fetched while the elements compute.
// The preconditioned residual of kPcg1 after the deferred update
//   s = w + beta s,  r = r - alpha s,  u = P r
// from the stored vectors; every place that needs u (the matvec's node stage,
// the node pass) forms it with this one function, so all agree bit for bit.
template <class S>
__device__ __forceinline__ V3<S> nextResidual(const Sys<S>& s, uint32_t n, S alpha, S beta, V3<S>& sOut, V3<S>& rOut) {
  sOut = fmaV(beta, xyz(ld4cg(&s.ap[n])), xyz(ld4cg(&s.w[n])));
  rOut = fmaV(-alpha, sOut, xyz(ld4cg(&s.r[n])));
  const Vec4<S> q0 = ld4g(&s.pre0[n]), q1 = ld4g(&s.pre1[n]);
  const Sym<S> P = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y};
  return symMul(P, rOut);
}

// Node values a tile's matvec multiplies: X if given; else (CGU) u, formed by
// nextResidual when `update` is set or read from z; else p = z + blend p_prev.
template <class S, bool CGU>
__device__ __forceinline__ V3<S> stagedValue(const Sys<S>& s, uint32_t n, const Vec4<S>* X, S blend, bool update,
                                             S alpha) {
  if (X) return xyz(ld4cg(&X[n]));
  if (CGU) {
    if (!update) return xyz(ld4cg(&s.z[n]));
    V3<S> so, ro;
    return nextResidual(s, n, alpha, blend, so, ro);
  }
  return fmaV(blend, xyz(ld4cg(&s.p[n])), xyz(ld4cg(&s.z[n])));
}

template <class S, int LAW, bool TANGENT, bool CGU = false, bool DAMP = false>
__device__ __forceinline__ void matvecTile(const Sys<S>& s, uint32_t tile, const Vec4<S>* X, S blend,
                                           S (*buf)[4 * TILE], uint16_t* sOff, uint16_t* sEnt, uint32_t elemEnd,
                                           bool update = false, S alpha = S(0)) {
  const uint32_t e = tile * TILE + threadIdx.x;
  const bool live = e < elemEnd;
  const uint2 meta = __ldg(&s.tile_meta[tile]);
  const uint2 entv = __ldg(reinterpret_cast<const uint2*>(s.tile_ent + size_t(tile) * 4 * TILE) + threadIdx.x);
  const uint16_t* off = s.tile_off + size_t(tile) * TILE_OFF_STRIDE;
  // only offsets 0..meta.y are read: fetch the 4-entry groups that hold them
  const uint2 offv = 4u * threadIdx.x <= meta.y ? __ldg(reinterpret_cast<const uint2*>(off) + threadIdx.x)
                                                : make_uint2(0u, 0u);
  const uint16_t offLast = threadIdx.x == 0 && meta.y >= 4u * TILE ? __ldg(&off[4 * TILE]) : uint16_t(0);
  const uint2 loc = live ? __ldg(&s.eloc[e]) : make_uint2(0u, 0u);
  // stage the tile's nodes: buf[k][j] = component k of node j
  for (uint32_t j = threadIdx.x; j < meta.y; j += TILE) {
    const uint32_t n = __ldg(&s.tile_node[meta.x + j]);
    const V3<S> v = stagedValue<S, CGU>(s, n, X, blend, update, alpha);
    buf[0][j] = v.x;
    buf[1][j] = v.y;
    buf[2][j] = v.z;
  }
  __syncthreads();
  V3<S> y[4] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  if (live) {
    const uint32_t l[4] = {loc.x & 0xffffu, loc.x >> 16, loc.y & 0xffffu, loc.y >> 16};
    V3<S> pe[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) pe[c] = {buf[0][l[c]], buf[1][l[c]], buf[2][l[c]]};
    elementApply<S, LAW, TANGENT, DAMP>(s, e, pe, y);
  }
  __syncthreads();  // node values consumed: buf now holds y, buf[k][c TILE + element]
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    buf[0][c * TILE + threadIdx.x] = y[c].x;
    buf[1][c * TILE + threadIdx.x] = y[c].y;
    buf[2][c * TILE + threadIdx.x] = y[c].z;
  }
  reinterpret_cast<uint2*>(sEnt)[threadIdx.x] = entv;
  reinterpret_cast<uint2*>(sOff)[threadIdx.x] = offv;
  if (threadIdx.x == 0) sOff[4 * TILE] = offLast;
  __syncthreads();
  for (uint32_t j = threadIdx.x; j < meta.y; j += TILE) {
    const uint32_t k0 = sOff[j], k1 = sOff[j + 1];
    S ax = 0, ay = 0, az = 0;
    for (uint32_t k = k0; k < k1; ++k) {
      const uint32_t code = sEnt[k];
      const uint32_t q = (code & 3u) * TILE + (code >> 2);
      ax += buf[0][q];
      ay += buf[1][q];
      az += buf[2][q];
    }
    s.slot_part[meta.x + j] = Vec4<S>{ax, ay, az, S(0)};
  }
  __syncthreads();
}

// Sum over node n's slots in ascending tile order, FP64 accumulation.  The
// first eight slot ids sit inline with the node (two 16-byte records), so all
// partial loads are issued at once; further slots come from the overflow CSR.
template <class S> __device__ __forceinline__ V3<double> gatherSlots(const Sys<S>& s, uint32_t n) {
  const uint4 i0 = __ldg(&s.ns_inline[n]), i1 = __ldg(&s.ns_inline[s.Vp + n]);
  const uint32_t k0 = __ldg(&s.ns_start[n]), k1 = __ldg(&s.ns_start[n + 1]);
  const uint32_t ids[8] = {i0.x, i0.y, i0.z, i0.w, i1.x, i1.y, i1.z, i1.w};
  Vec4<S> v[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) v[k] = ids[k] != NO_SLOT ? ld4cg(&s.slot_part[ids[k]]) : Vec4<S>{0, 0, 0, 0};
  V3<double> acc = {0, 0, 0};
#pragma unroll
  for (int k = 0; k < 8; ++k) acc = acc + cvt<double>(xyz(v[k]));
  for (uint32_t k = k0; k < k1; ++k) acc = acc + cvt<double>(xyz(ld4cg(&s.slot_part[__ldg(&s.ns_slot[k])])));
  return acc;
}

// Tile tables of one launch held in shared memory: a block of the
// single-body PCG always works the same tiles (blockIdx.x + k gridDim.x), so
// when it has at most CACHE_TILES of them it loads their local CSR, corner
// slots and node lists once per launch instead of once per iteration.
constexpr int CACHE_TILES = 4;
struct TileCache {
  uint2 meta[CACHE_TILES];
  uint16_t ent[CACHE_TILES][4 * TILE];
  uint16_t off[CACHE_TILES][TILE_OFF_STRIDE];
  uint2 eloc[CACHE_TILES][TILE];
  uint32_t node[CACHE_TILES][4 * TILE];
};

template <class S>
__device__ __forceinline__ void fillTileCache(const Sys<S>& s, TileCache& c, uint32_t tiles) {
  for (uint32_t k = 0; k < tiles; ++k) {
    const uint32_t tile = blockIdx.x + k * gridDim.x;
    const uint2 meta = __ldg(&s.tile_meta[tile]);
    if (threadIdx.x == 0) c.meta[k] = meta;
    reinterpret_cast<uint2*>(c.ent[k])[threadIdx.x] =
        __ldg(reinterpret_cast<const uint2*>(s.tile_ent + size_t(tile) * 4 * TILE) + threadIdx.x);
    const uint2* off = reinterpret_cast<const uint2*>(s.tile_off + size_t(tile) * TILE_OFF_STRIDE);
    for (uint32_t q = threadIdx.x; q < TILE_OFF_STRIDE / 4; q += TILE) reinterpret_cast<uint2*>(c.off[k])[q] = __ldg(off + q);
    c.eloc[k][threadIdx.x] = __ldg(&s.eloc[size_t(tile) * TILE + threadIdx.x]);
    for (uint32_t j = threadIdx.x; j < meta.y; j += TILE) c.node[k][j] = __ldg(&s.tile_node[meta.x + j]);
  }
  __syncthreads();
}

// matvecTile with the tile tables of cache entry k: the element operator is
// requested before the node stage, so the only dependent L2 round trip left
// is the node values.
template <class S, int LAW, bool TANGENT, bool CGU, bool DAMP>
__device__ __forceinline__ void matvecTileCached(const Sys<S>& s, const TileCache& c, uint32_t k, uint32_t tile,
                                                 const Vec4<S>* X, S blend, S (*buf)[4 * TILE], uint32_t elemEnd,
                                                 bool update, S alpha) {
  const uint32_t e = tile * TILE + threadIdx.x;
  const bool live = e < elemEnd;
  ElementOperator<S> op;
  if (live) op = loadOperator<S, LAW, TANGENT>(s, e);
  const uint2 meta = c.meta[k];
  for (uint32_t j = threadIdx.x; j < meta.y; j += TILE) {
    const V3<S> v = stagedValue<S, CGU>(s, c.node[k][j], X, blend, update, alpha);
    buf[0][j] = v.x;
    buf[1][j] = v.y;
    buf[2][j] = v.z;
  }
  __syncthreads();
  V3<S> y[4] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  if (live) {
    const uint2 loc = c.eloc[k][threadIdx.x];
    const uint32_t l[4] = {loc.x & 0xffffu, loc.x >> 16, loc.y & 0xffffu, loc.y >> 16};
    V3<S> pe[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) pe[q] = {buf[0][l[q]], buf[1][l[q]], buf[2][l[q]]};
    applyOperator<S, LAW, TANGENT>(op, pe, y);
    if (DAMP && LAW == 0) dampingProduct(s, e, op.g, pe, y);
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    buf[0][q * TILE + threadIdx.x] = y[q].x;
    buf[1][q * TILE + threadIdx.x] = y[q].y;
    buf[2][q * TILE + threadIdx.x] = y[q].z;
  }
  __syncthreads();
  for (uint32_t j = threadIdx.x; j < meta.y; j += TILE) {
    const uint32_t k0 = c.off[k][j], k1 = c.off[k][j + 1];
    S ax = 0, ay = 0, az = 0;
    for (uint32_t q = k0; q < k1; ++q) {
      const uint32_t code = c.ent[k][q];
      const uint32_t at = (code & 3u) * TILE + (code >> 2);
      ax += buf[0][at];
      ay += buf[1][at];
      az += buf[2][at];
    }
    s.slot_part[meta.x + j] = Vec4<S>{ax, ay, az, S(0)};
  }
  __syncthreads();
}

// Persistent PCG for a system holding ONE body: conjugateGradient
// (solver.cc:1904-2089, block-Jacobi branch) in the Chronopoulos-Gear
// arrangement, which needs one reduction per iteration instead of two.  The
// matvec is applied to u = P r rather than to p; p and s = A p follow by
// recurrence:
//   gamma = r.u, delta = u.A u, beta = gamma / gamma_prev,
//   p.A p = delta - beta gamma / alpha_prev, alpha = gamma / p.A p,
//   p = u + beta p, s = A u + beta s, x += alpha p, r -= alpha s, u = P r.
// In exact arithmetic the iterates equal the reference's; the stopping test
// (|r| <= tolerance |rhs| or the iteration cap, checked before each update),
// the breakdown test (p.A p > 0 and r.z > 0) and the iteration count are the
// reference's.  Per iteration:
//   A (element tiles)  A u_i, u_i formed on the fly from the update of the
//                      previous iteration (nextResidual), tile-local sums
//   B (node tiles)     apply that update (p, s, x, r, u), gather w = A u,
//                      partials of r.u, w.u, r.r
// with a grid barrier after each.  A solve that stops on the tolerance has
// computed one matvec more than the reference; one that reaches the cap
// finishes with a node pass that applies the last update without a matvec.
// Every block accumulates its partials in a fixed order and, after the
// barrier, adds all blocks' partials in block order, so every block takes the
// same decisions with no further communication.
template <class S, int LAW, bool TANGENT, bool DAMP = false>
__global__ void __launch_bounds__(TILE, sizeof(S) == 4 ? 3 : 2) kPcg1(Sys<S> s, Vec4<S>* X, uint32_t x0zero) {
  __shared__ S buf[3][4 * TILE];
  __shared__ __align__(8) uint16_t sOff[TILE_OFF_STRIDE];
  __shared__ __align__(8) uint16_t sEnt[4 * TILE];
  extern __shared__ __align__(16) unsigned char tlDyn[];  // TileCache
  TileCache& cache = *reinterpret_cast<TileCache*>(tlDyn);
  const uint32_t G = gridDim.x;
  const uint32_t perBlock = (s.elem_tiles + G - 1) / G;  // the same in every block
  const bool cached = perBlock <= uint32_t(CACHE_TILES);
  if (cached) fillTileCache(s, cache, blockIdx.x < s.elem_tiles ? (s.elem_tiles - 1 - blockIdx.x) / G + 1 : 0u);
  unsigned int bar = 0;
  const BodyDev bd = s.body[0];
  const BodyStepDev st = s.step[0];
  const S zero = S(0);
  double* part = s.blk_part;
  uint32_t applications = x0zero ? 0u : 1u;
  // ---- init: r = right - A x (anchored rows 0), u = P r, p = s = 0
  if (!x0zero) {
    for (uint32_t tile = blockIdx.x, k = 0; tile < s.elem_tiles; tile += G, ++k) {
      if (cached) matvecTileCached<S, LAW, TANGENT, true, DAMP>(s, cache, k, tile, X, zero, buf, bd.elem_end, false, zero);
      else matvecTile<S, LAW, TANGENT, false, DAMP>(s, tile, X, zero, buf, sOff, sEnt, bd.elem_end);
    }
    if (!countBarrier(s.sync, bar)) return;
  }
  {
    double rr = 0.0, bb = 0.0;
    for (uint32_t tile = blockIdx.x; tile < s.node_tiles; tile += G) {
      const uint32_t n = tile * TILE + threadIdx.x;
      if (n >= bd.node_end) continue;
      const Vec4<S> rhs = s.right[n];
      V3<S> r = {zero, zero, zero};
      if (!s.anch[n]) {
        V3<double> ax = {0, 0, 0};
        if (!x0zero) ax = (st.inertia * double(ld4g(&s.rest4[n]).w)) * cvt<double>(xyz(ld4cg(&X[n]))) + gatherSlots(s, n);
        r = cvt<S>(cvt<double>(xyz(rhs)) - ax);
      }
      const Vec4<S> q0 = s.pre0[n], q1 = s.pre1[n];
      const Sym<S> P = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y};
      s.r[n] = pack(r);
      s.z[n] = pack(symMul(P, r));
      s.p[n] = Vec4<S>{zero, zero, zero, zero};
      s.ap[n] = Vec4<S>{zero, zero, zero, zero};
      if (x0zero) X[n] = Vec4<S>{zero, zero, zero, zero};
      rr += dot(cvt<double>(r), cvt<double>(r));
      bb += dot(cvt<double>(xyz(rhs)), cvt<double>(xyz(rhs)));
    }
    double v[2] = {rr, bb};
    blockSum<2>(v);
    if (threadIdx.x == 0) {
      part[G + blockIdx.x] = v[0];
      part[2 * G + blockIdx.x] = v[1];
    }
  }
  if (!countBarrier(s.sync, bar)) return;
  double init[3];
  sumBlocksAll<3>(part, init);
  double length = init[1];
  const double reference = sqrt(init[2]);
  const double floor = fmax(reference, 1.1754943508222875e-38);  // std::numeric_limits<float>::min()
  const double target = st.tolerance * floor;
  const double startRes = sqrt(length) / floor;
  double gamma = 0.0, alpha = 0.0, beta = 0.0;
  uint32_t taken = 0;
  // apply the update with (alpha, beta) on this block's nodes; partial r.r
  auto applyUpdate = [&](double& rr) {
    for (uint32_t tile = blockIdx.x; tile < s.node_tiles; tile += G) {
      const uint32_t n = tile * TILE + threadIdx.x;
      if (n >= bd.node_end) continue;
      V3<S> sn, rn;
      const V3<S> un = nextResidual(s, n, S(alpha), S(beta), sn, rn);
      const V3<S> pn = fmaV(S(beta), xyz(ld4cg(&s.p[n])), xyz(ld4cg(&s.z[n])));
      X[n] = pack(fmaV(S(alpha), pn, xyz(ld4cg(&X[n]))));
      s.p[n] = pack(pn);
      s.ap[n] = pack(sn);
      s.r[n] = pack(rn);
      s.z[n] = pack(un);
      rr += dot(cvt<double>(rn), cvt<double>(rn));
    }
  };
  bool update = false;  // an update (alpha, beta) is pending
  if (!(taken >= st.limit || sqrt(length) <= target)) {
    for (;;) {
      // ---- A: w = A u
      for (uint32_t tile = blockIdx.x, k = 0; tile < s.elem_tiles; tile += G, ++k) {
        if (cached)
          matvecTileCached<S, LAW, TANGENT, true, DAMP>(s, cache, k, tile, nullptr, S(beta), buf, bd.elem_end,
                                                        update, S(alpha));
        else
          matvecTile<S, LAW, TANGENT, true, DAMP>(s, tile, nullptr, S(beta), buf, sOff, sEnt, bd.elem_end, update,
                                                  S(alpha));
      }
      ++applications;
      if (!countBarrier(s.sync, bar)) return;
      // ---- B: the pending update, w = inertia m u + sum of slots, partials
      double g = 0.0, d = 0.0, rr = 0.0;
      for (uint32_t tile = blockIdx.x; tile < s.node_tiles; tile += G) {
        const uint32_t n = tile * TILE + threadIdx.x;
        if (n >= bd.node_end) continue;
        V3<S> un, rn;
        if (update) {
          V3<S> sn;
          un = nextResidual(s, n, S(alpha), S(beta), sn, rn);
          const V3<S> pn = fmaV(S(beta), xyz(ld4cg(&s.p[n])), xyz(ld4cg(&s.z[n])));
          X[n] = pack(fmaV(S(alpha), pn, xyz(ld4cg(&X[n]))));
          s.p[n] = pack(pn);
          s.ap[n] = pack(sn);
          s.r[n] = pack(rn);
          s.z[n] = pack(un);
        } else {
          un = xyz(ld4cg(&s.z[n]));
          rn = xyz(ld4cg(&s.r[n]));
        }
        V3<S> wn = {zero, zero, zero};
        if (!s.anch[n]) wn = cvt<S>((st.inertia * double(ld4g(&s.rest4[n]).w)) * cvt<double>(un) + gatherSlots(s, n));
        s.w[n] = pack(wn);
        g += dot(cvt<double>(rn), cvt<double>(un));
        d += dot(cvt<double>(wn), cvt<double>(un));
        rr += dot(cvt<double>(rn), cvt<double>(rn));
      }
      {
        double v[3] = {g, d, rr};
        blockSum<3>(v);
        if (threadIdx.x == 0) {
          part[blockIdx.x] = v[0];
          part[G + blockIdx.x] = v[1];
          part[2 * G + blockIdx.x] = v[2];
        }
      }
      if (!countBarrier(s.sync, bar)) return;
      double sums[3];
      sumBlocksAll<3>(part, sums);
      const double gammaNext = sums[0], delta = sums[1];
      length = sums[2];
      if (update) {
        ++taken;
        if (taken >= st.limit || sqrt(length) <= target) break;  // the reference's loop-top test
      }
      const double b = update ? gammaNext / gamma : 0.0;
      const double curvature = update ? delta - b * gammaNext / alpha : delta;  // p.A p
      if (!(curvature > 0.0) || !(gammaNext > 0.0)) break;
      beta = b;
      alpha = gammaNext / curvature;
      gamma = gammaNext;
      update = true;
      if (taken + 1 >= st.limit) {  // the last update the cap allows: no matvec after it
        double rr2 = 0.0;
        applyUpdate(rr2);
        double v[1] = {rr2};
        blockSum<1>(v);
        if (threadIdx.x == 0) part[2 * G + blockIdx.x] = v[0];
        if (!countBarrier(s.sync, bar)) return;
        double fin[3];
        sumBlocksAll<3>(part, fin);
        length = fin[2];
        ++taken;
        break;
      }
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const double residual = sqrt(length);
    CgBodyDev c;
    c.squared = gamma;
    c.target = target;
    c.floor = floor;
    c.length = length;
    c.stride = alpha;
    c.blend = beta;
    c.start_res = startRes;
    c.rel_res = residual / floor;
    c.taken = taken;
    c.done = 1u;
    c.pad0 = c.pad1 = 0;
    s.cg[0] = c;
    CgReportDev rep = s.cgrep[0];
    rep.iterations += taken;
    rep.capped += (taken == st.limit && residual > target) ? 1u : 0u;
    rep.applications += applications;
    rep.solves += 1u;
    rep.tangent_iterations += TANGENT ? taken : 0u;
    rep.worst_rel = fmax(rep.worst_rel, c.rel_res);
    if (rep.pass_solves == 0u) rep.pass_start = c.start_res;
    rep.pass_end = c.rel_res;
    rep.pass_iterations += c.taken;
    rep.pass_solves += 1u;
    s.cgrep[0] = rep;
  }
}

// ---- software-pipelined tile loop of the batched PCG ----
// A block works through many tiles per phase.  While it computes tile k, its
// threads copy tile k+1's tables (local CSR, corner slots, node list) and
// element operators into the other half of a double-buffered shared stage
// (cp.async), and tile k+2's slot range comes into a register, so a tile
// waits for only one dependent L2/DRAM round trip: its node values.
struct TileTables {
  uint16_t ent[4 * TILE];
  uint16_t off[TILE_OFF_STRIDE];
  uint16_t pad[4];  // keeps the struct a multiple of 16 bytes
  uint2 eloc[TILE];
  uint32_t node[4 * TILE];
};
static_assert(sizeof(TileTables) % 16 == 0 && offsetof(TileTables, off) % 8 == 0 &&
                  offsetof(TileTables, eloc) % 8 == 0 && offsetof(TileTables, node) % 4 == 0,
              "cp.async destinations of the tile stage must stay aligned");
template <class S, int LAW, bool TANGENT> __host__ __device__ constexpr size_t pipeBytes() {
  return 2 * (sizeof(TileTables) + stageBytes<S, LAW, TANGENT>());
}
__device__ __forceinline__ void cpAsyncWaitNewest() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Queues the copies of one tile into a stage buffer (all threads take part).
template <class S, int LAW, bool TANGENT>
__device__ __forceinline__ void issueTile(const Sys<S>& s, uint32_t tile, uint2 meta, unsigned char* half) {
  TileTables& tt = *reinterpret_cast<TileTables*>(half);
  const uint32_t t = threadIdx.x, e = tile * TILE + t;  // e < Tp: padded elements have zeroed operators
  stageOperator<S, LAW, TANGENT>(s, e, half + sizeof(TileTables));
  cpAsync<8>(&tt.eloc[t], &s.eloc[e]);
  cpAsync<8>(&tt.ent[4 * t], s.tile_ent + size_t(tile) * 4 * TILE + 4 * t);
  const uint16_t* off = s.tile_off + size_t(tile) * TILE_OFF_STRIDE;
  if (4u * t <= meta.y) cpAsync<8>(&tt.off[4 * t], off + 4 * t);
  if (t == 0 && meta.y >= 4u * TILE) cpAsync<8>(&tt.off[4 * TILE], off + 4 * TILE);
  for (uint32_t j = t; j < meta.y; j += TILE) cpAsync<4>(&tt.node[j], s.tile_node + meta.x + j);
}

// The matvec of one staged tile (same arithmetic and order as matvecTile).
template <class S, int LAW, bool TANGENT, bool DAMP>
__device__ __forceinline__ void computeTile(const Sys<S>& s, uint32_t tile, uint2 meta, const unsigned char* half,
                                            const Vec4<S>* X, S blend, S (*buf)[4 * TILE], uint32_t elemEnd) {
  const TileTables& tt = *reinterpret_cast<const TileTables*>(half);
  const uint32_t e = tile * TILE + threadIdx.x;
  for (uint32_t j = threadIdx.x; j < meta.y; j += TILE) {
    const V3<S> v = stagedValue<S, false>(s, tt.node[j], X, blend, false, S(0));
    buf[0][j] = v.x;
    buf[1][j] = v.y;
    buf[2][j] = v.z;
  }
  __syncthreads();
  V3<S> y[4] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  if (e < elemEnd) {
    const uint2 loc = tt.eloc[threadIdx.x];
    const uint32_t l[4] = {loc.x & 0xffffu, loc.x >> 16, loc.y & 0xffffu, loc.y >> 16};
    V3<S> pe[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) pe[c] = {buf[0][l[c]], buf[1][l[c]], buf[2][l[c]]};
    const ElementOperator<S> op = stagedOperator<S, LAW, TANGENT>(half + sizeof(TileTables));
    applyOperator<S, LAW, TANGENT>(op, pe, y);
    if (DAMP && LAW == 0) dampingProduct(s, e, op.g, pe, y);
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    buf[0][c * TILE + threadIdx.x] = y[c].x;
    buf[1][c * TILE + threadIdx.x] = y[c].y;
    buf[2][c * TILE + threadIdx.x] = y[c].z;
  }
  __syncthreads();
  for (uint32_t j = threadIdx.x; j < meta.y; j += TILE) {
    const uint32_t k0 = tt.off[j], k1 = tt.off[j + 1];
    S ax = 0, ay = 0, az = 0;
    for (uint32_t k = k0; k < k1; ++k) {
      const uint32_t code = tt.ent[k];
      const uint32_t q = (code & 3u) * TILE + (code >> 2);
      ax += buf[0][q];
      ay += buf[1][q];
      az += buf[2][q];
    }
    s.slot_part[meta.x + j] = Vec4<S>{ax, ay, az, S(0)};
  }
  __syncthreads();
}

// Every tile of this block whose body takes part in the pass (and, when
// skipDone, has not converged), in order, pipelined.  X: multiply X instead
// of p = z + blend p_prev.  Done flags do not change during the phase.
template <class S, int LAW, bool TANGENT, bool DAMP>
__device__ __forceinline__ void matvecPipelined(const Sys<S>& s, uint32_t pass, const Vec4<S>* X, bool skipDone,
                                                unsigned char* dyn, S (*buf)[4 * TILE]) {
  constexpr uint32_t NONE = 0xffffffffu;
  constexpr size_t HALF = sizeof(TileTables) + stageBytes<S, LAW, TANGENT>();
  const uint32_t G = gridDim.x;
  auto next = [&](uint32_t t) -> uint32_t {
    for (; t < s.elem_tiles; t += G) {
      const uint32_t b = s.elem_tile_body[t];
      if (bodyActive(s, b, pass) && !(skipDone && __ldcg(&s.cg[b].done))) return t;
    }
    return NONE;
  };
  uint32_t t0 = next(blockIdx.x);
  if (t0 == NONE) return;
  uint2 m0 = __ldg(&s.tile_meta[t0]);
  uint32_t t1 = next(t0 + G);
  uint2 m1 = t1 != NONE ? __ldg(&s.tile_meta[t1]) : make_uint2(0u, 0u);
  issueTile<S, LAW, TANGENT>(s, t0, m0, dyn);
  cpAsyncCommit();
  for (uint32_t k = 0; t0 != NONE; ++k) {
    unsigned char* cur = dyn + (k & 1u) * HALF;
    if (t1 != NONE) issueTile<S, LAW, TANGENT>(s, t1, m1, dyn + ((k + 1u) & 1u) * HALF);
    cpAsyncCommit();
    const uint32_t t2 = t1 != NONE ? next(t1 + G) : NONE;
    const uint2 m2 = t2 != NONE ? __ldg(&s.tile_meta[t2]) : make_uint2(0u, 0u);
    cpAsyncWaitNewest();  // this thread's copies of tile t0 have landed
    __syncthreads();      // and everyone else's
    const uint32_t b0 = s.elem_tile_body[t0];
    const S blend = X ? S(0) : S(__ldcg(&s.cg[b0].blend));
    computeTile<S, LAW, TANGENT, DAMP>(s, t0, m0, cur, X, blend, buf, s.body[b0].elem_end);
    t0 = t1;
    m0 = m1;
    t1 = t2;
    m1 = m2;
  }
  cpAsyncWaitAll();
}

// Persistent PCG for a system of MANY bodies (the batched form): the phases of
// kPcg1 with the two-level assembly, but every body keeps its own scalars
// (CgBodyDev) and stops on its own test.  Per-tile partials are summed over a
// body's tiles, in tile order, by the block that finishes the body's last tile
// (lastTileOfBody); the launch ends when no body iterates.  Bodies that are
// done skip their tiles, so a batch costs the sum of its bodies' iterations,
// not bodies x the slowest body.
template <class S, int LAW, bool TANGENT, bool DAMP = false>
__global__ void __launch_bounds__(TILE, sizeof(S) == 4 ? 3 : 2)
    kPcgBatch(Sys<S> s, Vec4<S>* X, uint32_t pass, uint32_t x0zero) {
  __shared__ S buf[3][4 * TILE];
  extern __shared__ __align__(16) unsigned char tlStage[];  // pipeBytes<S, LAW, TANGENT>()
  const uint32_t G = gridDim.x;
  const S zero = S(0);
  unsigned int bar = 0;
  // ---- init: r = right - A x (anchored rows 0), z = P r, p_prev = 0
  if (!x0zero) {
    matvecPipelined<S, LAW, TANGENT, DAMP>(s, pass, X, false, tlStage, buf);
    if (!countBarrier(s.sync, bar)) return;
  }
  for (uint32_t tile = blockIdx.x; tile < s.node_tiles; tile += G) {
    const uint32_t b = s.node_tile_body[tile];
    if (!bodyActive(s, b, pass)) continue;
    const BodyDev bd = s.body[b];
    const uint32_t n = tile * TILE + threadIdx.x;
    double sums[3] = {0.0, 0.0, 0.0};
    if (n < bd.node_end) {
      const Vec4<S> rhs = s.right[n];
      V3<S> r = {zero, zero, zero};
      if (!s.anch[n]) {
        V3<double> ax = {0, 0, 0};
        if (!x0zero)
          ax = (s.step[b].inertia * double(ld4g(&s.rest4[n]).w)) * cvt<double>(xyz(ld4cg(&X[n]))) + gatherSlots(s, n);
        r = cvt<S>(cvt<double>(xyz(rhs)) - ax);
      }
      const Vec4<S> q0 = s.pre0[n], q1 = s.pre1[n];
      const Sym<S> P = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y};
      const V3<S> z = symMul(P, r);
      s.r[n] = pack(r);
      s.z[n] = pack(z);
      s.p[n] = Vec4<S>{zero, zero, zero, zero};
      if (x0zero) X[n] = Vec4<S>{zero, zero, zero, zero};
      sums[0] = dot(cvt<double>(r), cvt<double>(z));
      sums[1] = dot(cvt<double>(r), cvt<double>(r));
      sums[2] = dot(cvt<double>(xyz(rhs)), cvt<double>(xyz(rhs)));
    }
    blockSum<3>(sums);
    if (threadIdx.x == 0) {
      s.part[size_t(tile) * 4 + 0] = sums[0];
      s.part[size_t(tile) * 4 + 1] = sums[1];
      s.part[size_t(tile) * 4 + 2] = sums[2];
    }
    if (lastTileOfBody(&s.counter[b], bd.node_tile_end - bd.node_tile_begin)) {
      double tot[3];
      sumTiles<3>(s.part, bd.node_tile_begin, bd.node_tile_end, tot);
      if (threadIdx.x == 0) {
        CgBodyDev c;
        const double reference = sqrt(tot[2]);
        c.floor = fmax(reference, 1.1754943508222875e-38);  // std::numeric_limits<float>::min()
        c.target = s.step[b].tolerance * c.floor;
        c.squared = tot[0];
        c.length = tot[1];
        c.start_res = sqrt(tot[1]) / c.floor;
        c.rel_res = c.start_res;
        c.blend = 0.0;
        c.stride = 0.0;
        c.taken = 0;
        c.done = (s.step[b].limit == 0u || sqrt(c.length) <= c.target) ? 1u : 0u;
        c.pad0 = c.pad1 = 0;
        s.cg[b] = c;
        __threadfence();
        if (c.done) atomicSub(&s.sync->active, 1);
      }
    }
  }
  if (!countBarrier(s.sync, bar)) return;
  for (;;) {
    if (*(volatile int*)&s.sync->active <= 0) break;  // uniform: no block decrements between here and barrier A
    // ---- A
    matvecPipelined<S, LAW, TANGENT, DAMP>(s, pass, nullptr, true, tlStage, buf);
    if (!countBarrier(s.sync, bar)) return;
    // ---- B
    for (uint32_t tile = blockIdx.x; tile < s.node_tiles; tile += G) {
      const uint32_t b = s.node_tile_body[tile];
      if (!bodyActive(s, b, pass) || __ldcg(&s.cg[b].done)) continue;
      const BodyDev bd = s.body[b];
      const uint32_t n = tile * TILE + threadIdx.x;
      double sums[1] = {0.0};
      if (n < bd.node_end) {
        const S blend = S(__ldcg(&s.cg[b].blend));
        const V3<S> pn = fmaV(blend, xyz(ld4cg(&s.p[n])), xyz(ld4cg(&s.z[n])));
        s.p[n] = pack(pn);
        V3<S> apn = {zero, zero, zero};
        if (!s.anch[n]) apn = cvt<S>((s.step[b].inertia * double(ld4g(&s.rest4[n]).w)) * cvt<double>(pn) + gatherSlots(s, n));
        s.ap[n] = pack(apn);
        sums[0] = dot(cvt<double>(pn), cvt<double>(apn));
      }
      blockSum<1>(sums);
      if (threadIdx.x == 0) s.part[size_t(tile) * 4 + 3] = sums[0];
      if (lastTileOfBody(&s.counter[b], bd.node_tile_end - bd.node_tile_begin)) {
        double tot[1];
        sumTiles<1>(s.part + 3, bd.node_tile_begin, bd.node_tile_end, tot);
        if (threadIdx.x == 0) {
          const double curvature = tot[0];
          const double squared = __ldcg(&s.cg[b].squared);
          if (!(curvature > 0.0) || !(squared > 0.0)) {
            s.cg[b].done = 1u;
            __threadfence();
            atomicSub(&s.sync->active, 1);
          } else {
            s.cg[b].stride = squared / curvature;
            __threadfence();
          }
        }
      }
    }
    if (!countBarrier(s.sync, bar)) return;
    // ---- C
    for (uint32_t tile = blockIdx.x; tile < s.node_tiles; tile += G) {
      const uint32_t b = s.node_tile_body[tile];
      if (!bodyActive(s, b, pass) || __ldcg(&s.cg[b].done)) continue;
      const BodyDev bd = s.body[b];
      const uint32_t n = tile * TILE + threadIdx.x;
      double sums[2] = {0.0, 0.0};
      if (n < bd.node_end) {
        const S stride = S(__ldcg(&s.cg[b].stride));
        const V3<S> pn = xyz(ld4cg(&s.p[n]));
        const V3<S> x = fmaV(stride, pn, xyz(ld4cg(&X[n])));
        const V3<S> r = fmaV(-stride, xyz(ld4cg(&s.ap[n])), xyz(ld4cg(&s.r[n])));
        const Vec4<S> q0 = s.pre0[n], q1 = s.pre1[n];
        const Sym<S> P = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y};
        const V3<S> z = symMul(P, r);
        X[n] = pack(x);
        s.r[n] = pack(r);
        s.z[n] = pack(z);
        sums[0] = dot(cvt<double>(r), cvt<double>(z));
        sums[1] = dot(cvt<double>(r), cvt<double>(r));
      }
      blockSum<2>(sums);
      if (threadIdx.x == 0) {
        s.part[size_t(tile) * 4 + 0] = sums[0];
        s.part[size_t(tile) * 4 + 1] = sums[1];
      }
      if (lastTileOfBody(&s.counter[b], bd.node_tile_end - bd.node_tile_begin)) {
        double tot[2];
        sumTiles<2>(s.part, bd.node_tile_begin, bd.node_tile_end, tot);
        if (threadIdx.x == 0) {
          CgBodyDev c = loadCg(&s.cg[b]);
          c.blend = tot[0] / c.squared;
          c.squared = tot[0];
          c.length = tot[1];
          c.taken += 1u;
          c.done = (sqrt(c.length) <= c.target || c.taken >= s.step[b].limit) ? 1u : 0u;
          s.cg[b] = c;
          __threadfence();
          if (c.done) atomicSub(&s.sync->active, 1);
        }
      }
    }
    if (!countBarrier(s.sync, bar)) return;
  }
  if (blockIdx.x == 0) {
    for (uint32_t b = threadIdx.x; b < s.bodies; b += TILE) {
      if (!bodyActive(s, b, pass)) continue;
      CgBodyDev c = loadCg(&s.cg[b]);
      const double residual = sqrt(c.length);
      c.rel_res = residual / c.floor;
      s.cg[b].rel_res = c.rel_res;
      CgReportDev rep = s.cgrep[b];
      rep.iterations += c.taken;
      rep.capped += (c.taken == s.step[b].limit && residual > c.target) ? 1u : 0u;
      rep.applications += c.taken + (x0zero ? 0u : 1u);
      rep.solves += 1u;
      rep.tangent_iterations += TANGENT ? c.taken : 0u;
      rep.worst_rel = fmax(rep.worst_rel, c.rel_res);
      if (rep.pass_solves == 0u) rep.pass_start = c.start_res;
      rep.pass_end = c.rel_res;
      rep.pass_iterations += c.taken;
      rep.pass_solves += 1u;
      s.cgrep[b] = rep;
    }
  }
}

// Step constants chosen on the device (graph-captured steps): variants[2 b]
// holds body b's constants for the configured substeps, variants[2 b + 1] for
// the inverted-predictor substeps (solver.cc:3574-3583).  mode 0 takes the
// first (for the inversion test itself), mode 1 picks by the test's flag.
static __global__ void kStepSelect(BodyStepDev* step, const BodyStepDev* variants, const BodyAccDev* acc,
                                   uint32_t bodies, uint32_t mode) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= bodies) return;
  step[b] = variants[2 * b + ((mode == 1u && acc[b].inverts) ? 1u : 0u)];
}

// After substep `pass`: each active body's substep record from its report's
// pass fields, which are then cleared for the next substep.
template <class S>
__global__ void kSubstepRecord(Sys<S> s, SubstepRecordDev* records, uint32_t pass) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= s.bodies || !bodyActive(s, b, pass)) return;
  CgReportDev rep = s.cgrep[b];
  if (pass < SUBSTEP_RECORDS)
    records[size_t(b) * SUBSTEP_RECORDS + pass] = SubstepRecordDev{rep.pass_iterations, 0u, rep.pass_start, rep.pass_end};
  rep.pass_iterations = 0u;
  rep.pass_solves = 0u;
  rep.pass_start = 0.0;
  rep.pass_end = 0.0;
  s.cgrep[b] = rep;
}

// Clears the per-body step accumulators (min J key to its largest value).
static __global__ void kAccReset(BodyAccDev* acc, CgReportDev* rep, uint32_t bodies) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= bodies) return;
  BodyAccDev z;
  memset(&z, 0, sizeof(z));
  z.min_j_key = ~0ull;
  acc[b] = z;
  CgReportDev r;
  memset(&r, 0, sizeof(r));
  rep[b] = r;
}

// Resets the PCG launch state: active body count, tile counters, barrier
// arrivals.  The error word is left as it is: a wait that ran out in any solve
// of a step stays recorded until the host reads it at the step's end (the step
// clears it once, before its first launch), and later solves of the same step
// see it at their first barrier and leave at once.
template <class S>
__global__ void kPcgPrepare(Sys<S> s, uint32_t pass) {
  __shared__ int count;
  if (threadIdx.x == 0) count = 0;
  __syncthreads();
  for (uint32_t b = threadIdx.x; b < s.bodies; b += blockDim.x) {
    s.counter[b] = 0u;
    if (bodyActive(s, b, pass)) atomicAdd(&count, 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    s.sync->arrive = 0u;
    s.sync->active = count;
    s.sync->active_odd = count;
  }
}

// dst = src on the nodes of the gated bodies (or zero when src is null).
template <class S>
__global__ void __launch_bounds__(TILE) kNodeCopy(Sys<S> s, Vec4<S>* dst, const Vec4<S>* src, uint32_t pass) {
  const uint32_t tile = blockIdx.x, b = s.node_tile_body[tile];
  if (!bodyActive(s, b, pass)) return;
  const uint32_t n = tile * TILE + threadIdx.x;
  dst[n] = src ? src[n] : Vec4<S>{0, 0, 0, 0};
}

// Clears the per-body Newton acceptance maxima before kNewtonAccept.
static __global__ void kAccMovedReset(BodyAccDev* acc, uint32_t bodies) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= bodies) return;
  acc[b].moved_key = 0ull;
  acc[b].extent_key = 0ull;
}

// a += incr on free nodes (solver.cc:3941-3945).
template <class S>
__global__ void __launch_bounds__(TILE) kAddIncrement(Sys<S> s, Vec4<S>* target, uint32_t pass) {
  const uint32_t tile = blockIdx.x, b = s.node_tile_body[tile];
  if (!bodyActive(s, b, pass)) return;
  const uint32_t n = tile * TILE + threadIdx.x;
  if (n >= s.body[b].node_end || s.anch[n]) return;
  const Vec4<S> t = target[n], i = s.incr[n];
  target[n] = Vec4<S>{t.x + i.x, t.y + i.y, t.z + i.z, t.w};
}

// Newton acceptance (solver.cc:4091-4107): total += increment on free nodes,
// increment = 0 on anchored ones; max |increment| and max |x_evaluated|.
template <class S>
__global__ void __launch_bounds__(TILE) kNewtonAccept(Sys<S> s, uint32_t pass) {
  const uint32_t tile = blockIdx.x, b = s.node_tile_body[tile];
  if (!bodyActive(s, b, pass)) return;
  const uint32_t n = tile * TILE + threadIdx.x;
  unsigned long long moved = 0ull, extent = 0ull;
  if (n < s.body[b].node_end) {
    if (s.anch[n]) {
      s.incr[n] = Vec4<S>{0, 0, 0, 0};
    } else {
      const BodyStepDev& st = s.step[b];
      const V3<double> tot = cvt<double>(xyz(s.total[n]));
      const V3<double> inc = cvt<double>(xyz(s.incr[n]));
      V3<double> ev = cvt<double>(xyz(s.rest4[n])) + cvt<double>(xyz(s.weighted[n])) + st.scale * tot;
      if (st.floating) {  // frame positions are arms from the centre
        const FrameDev& f = s.frame[b];
        ev = ev - V3<double>{f.rest_centre[0], f.rest_centre[1], f.rest_centre[2]};
      }
      s.total[n] = packc<S>(tot + inc);
      moved = (unsigned long long)__double_as_longlong(sqrt(dot(inc, inc)));
      extent = (unsigned long long)__double_as_longlong(sqrt(dot(ev, ev)));
    }
  }
  moved = blockMaxKey(moved);
  extent = blockMaxKey(extent);
  if (threadIdx.x == 0) {
    atomicMax(&s.acc[b].moved_key, moved);
    atomicMax(&s.acc[b].extent_key, extent);
  }
}

// Backtrack (solver.cc:4061-4070): increment *= 1/2; total -= increment.
template <class S>
__global__ void __launch_bounds__(TILE) kBacktrack(Sys<S> s, uint32_t pass) {
  const uint32_t tile = blockIdx.x, b = s.node_tile_body[tile];
  if (!bodyActive(s, b, pass)) return;
  const uint32_t n = tile * TILE + threadIdx.x;
  if (n >= s.body[b].node_end) return;
  const Vec4<S> i = s.incr[n], t = s.total[n];
  const Vec4<S> h = {i.x * S(0.5), i.y * S(0.5), i.z * S(0.5), S(0)};
  s.incr[n] = h;
  s.total[n] = Vec4<S>{t.x - h.x, t.y - h.y, t.z - h.z, t.w};
}

// Velocity and position update (solver.cc:4350-4369, 5829-5849).  Anchored
// nodes move with their prescribed velocity (zero = the reference's fixed
// anchors).
template <class S>
__global__ void __launch_bounds__(TILE) kUpdate(Sys<S> s, uint32_t pass) {
  const uint32_t tile = blockIdx.x, b = s.node_tile_body[tile];
  if (!bodyActive(s, b, pass)) return;
  const uint32_t n = tile * TILE + threadIdx.x;
  if (n >= s.body[b].node_end) return;
  const BodyStepDev& st = s.step[b];
  if (st.floating) {
    // solver.cc:4325-4338, 5845-5847: the projection's spin corrections, then
    // the position.  kFrameEnd left the unconstrained velocity in v, the world
    // acceleration in a and the world arm in relv; restore and settle are
    // zero unless the split is Projected.
    const FrameDev& f = s.frame[b];
    const V3<double> arm = cvt<double>(xyz(s.relv[n]));
    const V3<double> turning = cross(V3<double>{f.settle[0], f.settle[1], f.settle[2]}, arm);
    const double spanned = st.beta * st.inner * st.inner;
    const V3<double> v = cvt<double>(xyz(s.v[n])) + cross(V3<double>{f.restore[0], f.restore[1], f.restore[2]}, arm);
    const V3<double> a = cvt<double>(xyz(s.a[n])) + turning;
    const V3<double> sh = cvt<double>(xyz(s.shifted[n])) - spanned * turning;
    s.v[n] = packc<S>(v);
    s.a[n] = packc<S>(a);
    s.u[n] = packc<S>(sh + spanned * a);
    return;
  }
  if (s.anch[n]) {
    const Vec4<S> pv = s.pres[n];
    s.v[n] = pv;
    s.a[n] = Vec4<S>{0, 0, 0, 0};
    const V3<double> u = cvt<double>(xyz(s.u[n])) + st.inner * cvt<double>(xyz(pv));
    s.u[n] = packc<S>(u);
    return;
  }
  const V3<double> a = cvt<double>(xyz(s.a[n]));
  const V3<double> v = cvt<double>(xyz(s.v[n])) + st.inner * ((1.0 - st.gamma) * cvt<double>(xyz(s.carried[n])) + st.gamma * a);
  const V3<double> u = cvt<double>(xyz(s.shifted[n])) + (st.beta * st.inner * st.inner) * a;
  s.v[n] = packc<S>(v);
  s.u[n] = packc<S>(u);
}

// Kinetic energy partials and the non-finite state check (solver.cc:5874-5879).
template <class S>
__global__ void __launch_bounds__(TILE) kStepEnd(Sys<S> s) {
  const uint32_t tile = blockIdx.x, b = s.node_tile_body[tile];
  const uint32_t n = tile * TILE + threadIdx.x;
  double ke = 0.0;
  bool bad = false;
  if (n < s.body[b].node_end) {
    const V3<double> v = cvt<double>(xyz(s.v[n]));
    const V3<double> u = cvt<double>(xyz(s.u[n])), a = cvt<double>(xyz(s.a[n]));
    ke = 0.5 * double(s.rest4[n].w) * dot(v, v);
    const bool finite = isfinite(u.x) && isfinite(u.y) && isfinite(u.z) && isfinite(v.x) && isfinite(v.y) &&
                        isfinite(v.z) && isfinite(a.x) && isfinite(a.y) && isfinite(a.z);
    bad = !finite;
  }
  const uint32_t nBad = blockCount(bad);
  if (threadIdx.x == 0 && nBad) atomicOr(&s.acc[b].nonfinite, 1u);
  double sums[1] = {ke};
  blockSum<1>(sums);
  if (threadIdx.x == 0) s.npart[size_t(tile) * 2 + 1] = sums[0];
}

}  // namespace tl
