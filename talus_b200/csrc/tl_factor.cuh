// tl_factor.cuh -- the caller-held Cholesky preconditioner on the device.
//
// A system with a solver state (DeformableSolverState, factor.h:205-210)
// preconditions its PCG with the FP64 factor of
//   A = (1 - alpha_m) M + h^2 sum_e R_e K_e R_e^T   (anchored rows: identity)
// made at the rotations and positions of its last refresh (SystemFactor,
// factor.cc:318-460, 567-618), applied in the frame that turns the body from
// those positions to the current ones (applyFactor, factor.cc:669-704;
// bodyRotation, factor.cc:620-667).  The factor is L with P A P^T = L L^T
// in 3x3 node blocks under a nested-dissection order P, made on the host.
//
// Kernels:
//   kFactorFrame  (one block) the body rotation: polar of the mass-weighted
//                 correlation of the positions now with the factor's
//   kPcgFactor    persistent cooperative PCG in the reference's order with
//                 the factor as preconditioner, operator = the assembled block
//                 matrix of kSellAssemble.  The two triangular solves of each
//                 application run inside the launch over the supernodes of the
//                 dissection (its leaves and separators): every block takes
//                 supernodes by an atomic ticket, children before parents in
//                 the forward solve and parents before children in the
//                 backward one, and waits (bounded) for the flags of the
//                 supernodes it reads.  Supernodes are handed out only to
//                 running blocks in dependency order, so the smallest
//                 unfinished ticket can always finish.
#pragma once

#include "tl_sell.cuh"

namespace tl {

// The factor in the layout of the two triangular solves, FP64.
struct FactorDev {
  uint32_t nodes;
  const uint32_t* perm;       // [nodes] factor order -> node
  const uint32_t* iperm;      // [nodes] node -> factor order
  const uint32_t* row_start;  // [nodes + 1] strictly lower blocks of row i of L
  const uint32_t* row_col;    // [row blocks] their columns
  const double* row_blk;      // [9 per block] L_ij row-major
  const uint32_t* col_start;  // [nodes + 1] strictly lower blocks of column i of L
  const uint32_t* col_row;    // [col blocks] their rows
  const double* col_blk;      // [9 per block] L_ji row-major
  const double* diag_inv;     // [9 per node] L_ii^-1 row-major (lower triangular)
  uint32_t supernodes;
  const uint32_t* sn_start;   // [supernodes + 1] row range of each supernode (children first)
  const int32_t* sn_child;    // [2 per supernode] -1: none
  const int32_t* sn_parent;   // [supernodes] -1: a root
  const uint32_t* row_split;  // [nodes] first block of row i inside its supernode
  const uint32_t* col_split;  // [nodes] first block of column i past its supernode
  Vec4<double>* rhs;          // [nodes] right sides less the finished supernodes' part
  Vec4<double>* y;            // [nodes] forward solve
  Vec4<double>* w;            // [nodes] backward solve
  uint32_t* fwd_flag;         // [supernodes] application epoch of the supernode's y
  uint32_t* bwd_flag;         // [supernodes] application epoch of the supernode's w
  uint32_t* ticket;           // [3] supernode tickets, by application mod 3
  uint32_t* epoch;            // [1] applications made so far (flags start at 0)
  const double* frame;        // [9] row-major rotation the factor is applied in
  double* part;               // [8 G] block partials, two halves
};

__device__ __forceinline__ void stRelease(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ uint32_t ldRelaxed(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Waits until flags[j[0..n)] (n <= FLAG_BATCH supernodes) all hold epoch:
// every pending flag is polled at once with relaxed loads, then one acquire
// fence orders the reads of those supernodes' values after them.  Bounded:
// gives up after TL_BARRIER_LIMIT_NS (recording TL_ERR_TIMEOUT) or once
// another wait or barrier has given up.
constexpr int FLAG_BATCH = 8;
__device__ __forceinline__ bool waitFlags(const uint32_t* flags, const uint32_t (&j)[FLAG_BATCH], uint32_t n,
                                          uint32_t epoch, GridSyncDev* sync) {
  uint32_t pending = n >= 32u ? 0xffffffffu : (1u << n) - 1u;
  unsigned long long t0 = 0;
  unsigned int rounds = 0;
  for (;;) {
#pragma unroll
    for (int b = 0; b < FLAG_BATCH; ++b)
      if ((pending >> b) & 1u)
        if (ldRelaxed(&flags[j[b]]) == epoch) pending &= ~(1u << b);
    if (!pending) break;
    if (rounds == 0) t0 = globalTimer();
    if ((++rounds & 63u) == 0u) {
      if (*(volatile int*)&sync->error != 0) return false;
      if (globalTimer() - t0 > TL_BARRIER_LIMIT_NS) {
        atomicExch(&sync->error, 5);  // TL_ERR_TIMEOUT
        return false;
      }
    }
    __nanosleep(32);
  }
  asm volatile("fence.acq_rel.gpu;" ::: "memory");
  return true;
}

__device__ __forceinline__ V3<double> warpSum3(V3<double> v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    v.z += __shfl_xor_sync(0xffffffffu, v.z, o);
  }
  return v;
}

// Sum of a V3 over the block; the result in thread 0.
__device__ __forceinline__ V3<double> blockSum3(V3<double> v, double (&red)[3][TILE / 32]) {
  v = warpSum3(v);
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][warp] = v.x;
    red[1][warp] = v.y;
    red[2][warp] = v.z;
  }
  __syncthreads();
  V3<double> sum = {0, 0, 0};
  if (threadIdx.x == 0)
    for (int w = 0; w < TILE / 32; ++w) sum = sum + V3<double>{red[0][w], red[1][w], red[2][w]};
  return sum;
}

// Rows of a supernode whose solved values a block keeps in shared memory
// (later rows of larger supernodes read theirs from global memory).
constexpr uint32_t SN_CACHE = 1024;

// z = frame (L L^T)^-1 P (frame^T r) of applyFactor, y and w in factor order;
// every block of the grid takes part.  Blocks take supernodes by an atomic
// ticket: the forward solve's in increasing order (children first), each
// after its children's flags; then the backward solve's in decreasing order
// (parents first), each after its parent's flag (a root: after its own
// forward flag, which follows every descendant's).  A block first takes the
// finished supernodes' part of all its rows at once (a warp per row), then
// solves its rows one after another, all threads on each row's blocks inside
// the supernode, the values solved so far in shared memory.  r is read at the
// forward rows (written before the launch's last grid barrier); the caller
// turns w back.
template <class S>
__device__ void factorSolve(const FactorDev& f, GridSyncDev* sync, const Vec4<S>* r, const M3<S>& frame,
                            uint32_t epoch, uint32_t* ticket) {
  __shared__ uint32_t snTicket;
  __shared__ double red[3][TILE / 32];
  __shared__ double solved[3][SN_CACHE];
  __shared__ uint32_t span[2][SN_CACHE];  // each cached row's own blocks [k0, k1)
  const uint32_t SN = f.supernodes, lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  bool ok = true;
  for (;;) {
    if (threadIdx.x == 0) snTicket = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint32_t t = snTicket;
    if (t >= 2u * SN) break;
    const bool forward = t < SN;
    const uint32_t p = forward ? t : 2u * SN - 1u - t;
    if (threadIdx.x == 0) {  // the supernodes this one reads
      uint32_t wait[FLAG_BATCH] = {0, 0, 0, 0, 0, 0, 0, 0};
      uint32_t n = 0;
      if (forward) {
        for (int c = 0; c < 2; ++c) {
          const int32_t ch = __ldg(&f.sn_child[2 * p + c]);
          if (ch >= 0) wait[n++] = uint32_t(ch);
        }
        ok = ok && waitFlags(f.fwd_flag, wait, n, epoch, sync);
      } else {
        const int32_t parent = __ldg(&f.sn_parent[p]);
        wait[0] = parent >= 0 ? uint32_t(parent) : p;
        ok = ok && waitFlags(parent >= 0 ? f.bwd_flag : f.fwd_flag, wait, 1u, epoch, sync);
      }
    }
    __syncthreads();
    const uint32_t b = __ldg(&f.sn_start[p]), e = __ldg(&f.sn_start[p + 1]);
    const uint32_t* start = forward ? f.row_start : f.col_start;
    const uint32_t* index = forward ? f.row_col : f.col_row;
    const Vec4<double>* val = forward ? f.y : f.w;
    const double* blk = forward ? f.row_blk : f.col_blk;
    // forward: L_ij v; backward: L_ji^T v (L row-major, in registers)
    const auto termR = [&](const double (&L)[9], const Vec4<double>& v, V3<double>& acc) {
      if (forward) {
        acc.x += L[0] * v.x + L[1] * v.y + L[2] * v.z;
        acc.y += L[3] * v.x + L[4] * v.y + L[5] * v.z;
        acc.z += L[6] * v.x + L[7] * v.y + L[8] * v.z;
      } else {
        acc.x += L[0] * v.x + L[3] * v.y + L[6] * v.z;
        acc.y += L[1] * v.x + L[4] * v.y + L[7] * v.z;
        acc.z += L[2] * v.x + L[5] * v.y + L[8] * v.z;
      }
    };
    const auto term = [&](const double* Lg, const Vec4<double>& v, V3<double>& acc) {
      double L[9];
#pragma unroll
      for (int m = 0; m < 9; ++m) L[m] = __ldg(Lg + m);
      termR(L, v, acc);
    };
    // ---- the finished supernodes' part of every row: forward the blocks
    // before the supernode, backward those past it; rhs = b_i - that part
    for (uint32_t i = b + warp; i < e; i += TILE / 32) {
      const uint32_t k0 = forward ? __ldg(&start[i]) : __ldg(&f.col_split[i]);
      const uint32_t k1 = forward ? __ldg(&f.row_split[i]) : __ldg(&start[i + 1]);
      if (lane == 0 && i - b < SN_CACHE) {  // the blocks inside the supernode, for the solve below
        span[0][i - b] = forward ? k1 : __ldg(&start[i]);
        span[1][i - b] = forward ? __ldg(&start[i + 1]) : k0;
      }
      V3<double> acc = {0, 0, 0};
      // a warp per row, several of each lane's blocks in flight at once
      uint32_t k = k0 + lane;
      for (; k + 96u < k1; k += 128u) {
        uint32_t jj[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) jj[u] = __ldg(&index[k + 32u * u]);
        Vec4<double> vv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) vv[u] = ld4cg(&val[jj[u]]);
#pragma unroll
        for (int u = 0; u < 4; ++u) term(blk + size_t(9) * (k + 32u * u), vv[u], acc);
      }
      for (; k < k1; k += 32u) term(blk + size_t(9) * k, ld4cg(&val[__ldg(&index[k])]), acc);
      acc = warpSum3(acc);
      if (lane == 0) {
        V3<double> rhs;
        if (forward) {  // frame^T r in the step's arithmetic
          rhs = cvt<double>(mulT(frame, xyz(ld4cg(&r[__ldg(&f.perm[i])]))));
        } else {
          const Vec4<double> yi = ld4cg(&f.y[i]);
          rhs = {yi.x, yi.y, yi.z};
        }
        f.rhs[i] = Vec4<double>{rhs.x - acc.x, rhs.y - acc.y, rhs.z - acc.z, 0.0};
      }
    }
    __syncthreads();
    // ---- the supernode's own rows in order.  Each row's first block per
    // thread, its L_ii^-1 and right side are requested while the row before
    // it is reduced, so a row costs its reduction and two block barriers.
    const auto rowOf = [&](uint32_t q) { return forward ? b + q : e - 1u - q; };
    const auto spanOf = [&](uint32_t q, uint32_t& k0, uint32_t& k1) {
      const uint32_t i = rowOf(q);
      if (i - b < SN_CACHE) {
        k0 = span[0][i - b];
        k1 = span[1][i - b];
      } else {
        k0 = forward ? __ldg(&f.row_split[i]) : __ldg(&start[i]);
        k1 = forward ? __ldg(&start[i + 1]) : __ldg(&f.col_split[i]);
      }
    };
    uint32_t nj = 0, nk = 0;
    bool nvalid = false;
    double nL[9], nd[9];
    Vec4<double> nrhs = {0, 0, 0, 0};
    const auto fetch = [&](uint32_t q) {  // requests for row q
      uint32_t k0, k1;
      spanOf(q, k0, k1);
      nk = k0 + threadIdx.x;
      nvalid = nk < k1;
      if (nvalid) {
        nj = __ldg(&index[nk]);
#pragma unroll
        for (int m = 0; m < 9; ++m) nL[m] = __ldg(blk + size_t(9) * nk + m);
      }
      if (threadIdx.x == 0) {
        const double* D = f.diag_inv + size_t(9) * rowOf(q);
#pragma unroll
        for (int m = 0; m < 9; ++m) nd[m] = __ldg(D + m);
        nrhs = ld4cg(&f.rhs[rowOf(q)]);
      }
    };
    if (e > b) fetch(0);
    for (uint32_t q = 0; q < e - b; ++q) {
      const uint32_t i = rowOf(q);
      uint32_t k0, k1;
      spanOf(q, k0, k1);
      const bool valid = nvalid;
      const uint32_t j0 = nj;
      double L0[9], d[9];
#pragma unroll
      for (int m = 0; m < 9; ++m) {
        L0[m] = nL[m];
        d[m] = nd[m];
      }
      const Vec4<double> rhs = nrhs;
      const auto value = [&](uint32_t j) {
        const uint32_t at = j - b;
        return at < SN_CACHE ? Vec4<double>{solved[0][at], solved[1][at], solved[2][at], 0.0} : ld4cg(&val[j]);
      };
      V3<double> acc = {0, 0, 0};
      if (valid) termR(L0, value(j0), acc);
      // the thread's further blocks of the row, four at a time with their
      // loads issued together
      uint32_t k = k0 + threadIdx.x + TILE;
      for (; k + 3u * TILE < k1; k += 4u * TILE) {
        uint32_t jj[4];
        double Lq[4][9];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          jj[u] = __ldg(&index[k + u * TILE]);
#pragma unroll
          for (int m = 0; m < 9; ++m) Lq[u][m] = __ldg(blk + size_t(9) * (k + u * TILE) + m);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) termR(Lq[u], value(jj[u]), acc);
      }
      for (; k < k1; k += TILE) term(blk + size_t(9) * k, value(__ldg(&index[k])), acc);
      if (q + 1 < e - b) fetch(q + 1);
      const V3<double> sum = blockSum3(acc, red);
      if (threadIdx.x == 0) {
        const V3<double> bb = {rhs.x - sum.x, rhs.y - sum.y, rhs.z - sum.z};
        const V3<double> x = forward ? V3<double>{d[0] * bb.x, d[3] * bb.x + d[4] * bb.y,
                                                  d[6] * bb.x + d[7] * bb.y + d[8] * bb.z}   // L_ii^-1 bb
                                     : V3<double>{d[0] * bb.x + d[3] * bb.y + d[6] * bb.z,  // L_ii^-T bb
                                                  d[4] * bb.y + d[7] * bb.z, d[8] * bb.z};
        (forward ? f.y : f.w)[i] = Vec4<double>{x.x, x.y, x.z, 0.0};
        if (i - b < SN_CACHE) {
          solved[0][i - b] = x.x;
          solved[1][i - b] = x.y;
          solved[2][i - b] = x.z;
        }
      }
      __syncthreads();  // the row is visible to the block's next rows; red is free again
    }
    if (threadIdx.x == 0) stRelease(forward ? &f.fwd_flag[p] : &f.bwd_flag[p], epoch);
  }
  (void)ok;  // a wait that gave up has recorded it; the next grid barrier ends the launch
}

// bodyRotation (factor.cc:620-667) of one body (nodes [0, V)): the polar
// rotation of sum_n m_n (x_n - c)(x0_n - c0)^T, x = rest + u now, x0 the
// positions at the refresh and c, c0 the mass-weighted centres.  One block.
template <class S>
__global__ void __launch_bounds__(TILE) kFactorFrame(Sys<S> s, uint32_t V, const Vec4<double>* ref, double* frame) {
  __shared__ double centre[3];
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  for (uint32_t n = threadIdx.x; n < V; n += TILE) {
    const Vec4<S> r4 = s.rest4[n], u = s.u[n];
    const double m = double(r4.w);
    v[0] += m;
    v[1] += m * (double(r4.x) + double(u.x));
    v[2] += m * (double(r4.y) + double(u.y));
    v[3] += m * (double(r4.z) + double(u.z));
  }
  blockSum<4>(v);
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; ++k) centre[k] = v[0] > 0.0 ? v[k + 1] / v[0] : v[k + 1];
  __syncthreads();
  // ref[V] holds the centre of the refresh positions
  const Vec4<double> c0 = ref[V];
  double c[9];
  for (int k = 0; k < 9; ++k) c[k] = 0.0;
  for (uint32_t n = threadIdx.x; n < V; n += TILE) {
    const Vec4<S> r4 = s.rest4[n], u = s.u[n];
    const Vec4<double> x0 = ref[n];
    const double m = double(r4.w);
    const double now[3] = {double(r4.x) + double(u.x) - centre[0], double(r4.y) + double(u.y) - centre[1],
                           double(r4.z) + double(u.z) - centre[2]};
    const double before[3] = {x0.x - c0.x, x0.y - c0.y, x0.z - c0.z};
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) c[3 * i + j] += m * now[i] * before[j];
  }
  blockSum<9>(c);
  if (threadIdx.x == 0) {
    M3<double> corr;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) corr.m[i][j] = c[3 * i + j];
    const M3<double> rot = polarRotation(corr);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) frame[3 * i + j] = rot.m[i][j];
  }
}

// Sum of N doubles over the grid: block partials into half `h` of part, a
// grid barrier, then the same block-ordered sum in every block.
template <int N>
__device__ __forceinline__ bool gridSum(double (&v)[N], double* part, uint32_t& h, GridSyncDev* sync,
                                        unsigned int& bar, double (&out)[N]) {
  double* half = part + size_t(4) * gridDim.x * (h++ & 1u);
  blockSum<N>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < N; ++k) half[size_t(k) * gridDim.x + blockIdx.x] = v[k];
  if (!countBarrier(sync, bar)) return false;
  sumBlocksAll<N>(half, out);
  return true;
}

// Persistent PCG of one body preconditioned by the factor (conjugateGradient,
// solver.cc:1904-2089, with condition = applyFactor): the reference's order,
// loop-top stopping test, breakdown test and cap.  Vectors live in global
// memory (x in X; r, d, q, z in the four planes given); rows are the
// assembled matrix's, a warp per 32-row slice, grid-strided; dots are FP64.
template <class S>
__global__ void __launch_bounds__(TILE) kPcgFactor(Sys<S> s, SellDev<S> g, FactorDev f, Vec4<S>* X, Vec4<S>* R,
                                                   Vec4<S>* D, Vec4<S>* Q, Vec4<S>* Z, uint32_t x0zero, uint32_t limit) {
  const uint32_t warps = gridDim.x * (TILE / 32u), gw = blockIdx.x * (TILE / 32u) + (threadIdx.x >> 5);
  const uint32_t lane = threadIdx.x & 31u;
  const BodyStepDev st = s.step[0];
  g.col_cache = 0;  // columns from global memory
  M3<S> frame;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) frame.m[i][j] = S(__ldcg(&f.frame[3 * i + j]));
  const uint32_t epoch0 = __ldcg(f.epoch);
  if (blockIdx.x == 0 && threadIdx.x < 3) f.ticket[threadIdx.x] = 0u;
  unsigned int bar = 0;
  uint32_t h = 0, apps = 0;
  // the rows of this thread: slices gw, gw + warps, ...; lane = row in slice
  auto forRows = [&](auto&& fn) {
    for (uint32_t slice = gw; slice < g.slices; slice += warps) {
      const uint32_t row = slice * SELL_ROWS + lane;
      fn(slice, row, row < g.rows && !s.anch[row], row < g.rows);
    }
  };
  auto matvec = [&](uint32_t slice, const Vec4<S>* in) {
    return sellRowOf<S, Ld4cg<S>, sellRowGroup<S>(), false>(g, slice, lane, ld4cgOf(in), nullptr);
  };
  // one application: z = frame (LL^T)^-1 frame^T r, anchored rows zero
  auto condition = [&](double& rz, double& rr) -> bool {
    if (blockIdx.x == 0 && threadIdx.x == 0) f.ticket[(apps + 1u) % 3u] = 0u;
    factorSolve<S>(f, s.sync, R, frame, epoch0 + apps + 1u, &f.ticket[apps % 3u]);
    ++apps;
    if (!countBarrier(s.sync, bar)) return false;
    rz = 0.0;
    rr = 0.0;
    forRows([&](uint32_t, uint32_t row, bool freeRow, bool live) {
      if (!live) return;
      V3<S> z = {0, 0, 0};
      if (freeRow) {
        const Vec4<double> w = ld4cg(&f.w[__ldg(&f.iperm[row])]);
        z = mul(frame, V3<S>{S(w.x), S(w.y), S(w.z)});
      }
      Z[row] = pack(z);
      const V3<double> r = cvt<double>(xyz(R[row])), zd = cvt<double>(z);
      rz += dot(r, zd);
      rr += dot(r, r);
    });
    return true;
  };
  // ---- r = right - A x (anchored rows 0), |right|
  double v0[1] = {0.0};
  forRows([&](uint32_t slice, uint32_t row, bool freeRow, bool live) {
    V3<double> r = {0, 0, 0};
    const V3<double> rhs = live ? cvt<double>(xyz(s.right[row])) : V3<double>{0, 0, 0};
    if (x0zero) {
      if (live) X[row] = Vec4<S>{0, 0, 0, 0};
      if (freeRow) r = rhs;
    } else {
      const V3<double> ax = matvec(slice, X);
      if (freeRow) r = rhs - ax;
    }
    if (live) {
      R[row] = pack(cvt<S>(r));
      v0[0] += dot(rhs, rhs);
    }
  });
  double refSq[1];
  if (!gridSum<1>(v0, f.part, h, s.sync, bar, refSq)) return;
  const double reference = sqrt(refSq[0]);
  double rz = 0.0, rr = 0.0;
  if (!condition(rz, rr)) return;
  forRows([&](uint32_t, uint32_t row, bool, bool live) {
    if (live) D[row] = Z[row];
  });
  double v1[2] = {rz, rr}, s1[2];
  if (!gridSum<2>(v1, f.part, h, s.sync, bar, s1)) return;
  double squared = s1[0], length = s1[1];
  const double floor = fmax(reference, 1.1754943508222875e-38);  // std::numeric_limits<float>::min()
  const double target = st.tolerance * floor;
  const double startRes = sqrt(length) / floor;
  double stride = 0.0, blend = 0.0;
  uint32_t taken = 0;
  for (uint32_t iteration = 0; iteration != limit; ++iteration) {
    if (sqrt(length) <= target) break;
    double vc[1] = {0.0}, curv[1];
    forRows([&](uint32_t slice, uint32_t row, bool freeRow, bool live) {
      const V3<double> q = matvec(slice, D);
      if (!live) return;
      const V3<S> qs = freeRow ? cvt<S>(q) : V3<S>{0, 0, 0};
      Q[row] = pack(qs);
      vc[0] += dot(cvt<double>(xyz(D[row])), cvt<double>(qs));
    });
    if (!gridSum<1>(vc, f.part, h, s.sync, bar, curv)) return;
    if (!(curv[0] > 0.0) || !(squared > 0.0)) break;
    stride = squared / curv[0];
    forRows([&](uint32_t, uint32_t row, bool, bool live) {
      if (!live) return;
      const V3<double> d = cvt<double>(xyz(D[row]));
      X[row] = pack(cvt<S>(cvt<double>(xyz(X[row])) + stride * d));
      R[row] = pack(cvt<S>(cvt<double>(xyz(R[row])) - stride * cvt<double>(xyz(Q[row]))));
    });
    if (!countBarrier(s.sync, bar)) return;
    if (!condition(rz, rr)) return;
    double vn[2] = {rz, rr}, sn[2];
    if (!gridSum<2>(vn, f.part, h, s.sync, bar, sn)) return;
    blend = sn[0] / squared;
    squared = sn[0];
    length = sn[1];
    forRows([&](uint32_t, uint32_t row, bool, bool live) {
      if (!live) return;
      D[row] = pack(cvt<S>(cvt<double>(xyz(Z[row])) + blend * cvt<double>(xyz(D[row]))));
    });
    ++taken;
    if (!countBarrier(s.sync, bar)) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const double residual = sqrt(length);
    CgBodyDev c;
    c.squared = squared;
    c.target = target;
    c.floor = floor;
    c.length = length;
    c.stride = stride;
    c.blend = blend;
    c.start_res = startRes;
    c.rel_res = residual / floor;
    c.taken = taken;
    c.done = 1u;
    c.pad0 = (taken == limit && residual > target) ? 1u : 0u;  // capped
    c.pad1 = apps;                                               // factor applications
    s.cg[0] = c;
    *f.epoch = epoch0 + apps;
  }
}

// The report of a finished factored solve (the recordCg of solver.cc:3621-3637
// for the result solvePrimary returns), as kPcgSell writes it.
template <class S>
__global__ void kFactorRecord(Sys<S> s, uint32_t tangent) {
  const CgBodyDev c = s.cg[0];
  CgReportDev rep = s.cgrep[0];
  rep.iterations += c.taken;
  rep.capped += c.pad0;
  rep.applications += c.taken + 1u;
  rep.solves += 1u;
  rep.tangent_iterations += tangent ? c.taken : 0u;
  rep.worst_rel = fmax(rep.worst_rel, c.rel_res);
  if (rep.pass_solves == 0u) rep.pass_start = c.start_res;
  rep.pass_end = c.rel_res;
  rep.pass_iterations += c.taken;
  rep.pass_solves += 1u;
  s.cgrep[0] = rep;
}

}  // namespace tl
