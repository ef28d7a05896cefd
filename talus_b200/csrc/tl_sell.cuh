// PCG on the assembled operator.
//
// The element-by-element matvec of kPcg1 spends most of each iteration
// moving element outputs back to the nodes through shared memory (bank
// conflicts, warp divergence) and needs a grid barrier between the element
// and the node phases.  Within one PCG solve the operator is fixed, so this
// path assembles it once per solve into 3x3 node blocks (the sum over the
// elements sharing two nodes of their h_eff^2 R K R^T blocks, plus
// (1 - alpha_m) m I on the diagonal, solver.cc:904-1048) and runs the solve
// on that matrix:
//
//   kSellAssemble  one thread per block above the diagonal: the sum,
//                  in ascending element order, of the element blocks that
//                  land there (FP64 accumulation, stored in S), written with
//                  its transpose below the diagonal; the diagonal blocks are
//                  written by kNodeAssemble;
//   kPcgBatchSell  the batched PCG on this matrix, for batches and for
//                  single bodies with more rows than kPcgSell's grid has
//                  threads, in the textbook order (two grid barriers per
//                  iteration): the order of FP32-mixed systems;
//   kPcgBatchSellPipe  the same solve in kPcgSell's pipelined arrangement
//                  with per-body scalars, one grid barrier per iteration and
//                  its recurrences in FP64: the order of FP64 systems;
//   kPcgSell       (one body) persistent cooperative PCG in the pipelined arrangement
//                  of Ghysels and Vanroose ("Hiding global synchronization
//                  latency in the preconditioned conjugate gradient
//                  algorithm", 2014), which overlaps the one reduction of an
//                  iteration with its matvec, so each iteration needs one grid
//                  barrier.  Each thread owns one node row and keeps its
//                  vectors in FP64 registers; only the matvec input is
//                  published (rounded to S, and used rounded on both sides).
//
// Layout: sliced ELL with 32 rows per slice (one warp).  Slice s holds its
// rows' blocks in width_s columns; block position p = slice_start[s] +
// 32 k + lane is column slot k of row 32 s + lane, and its 9 entries sit at
// val[(p >> 5) 288 + 32 c + lane], so a warp reads each entry of 32 rows in
// one 128-byte (FP32) transaction.  Column slots are the row's neighbour
// nodes in ascending order; a row with fewer neighbours than its slice's
// width pads with zero blocks on its own column.
#pragma once

#include "tl_kernels.cuh"
#include "tl_sell_build.h"

namespace tl {

constexpr uint32_t SELL_SLICES_PER_BLOCK = TILE / SELL_ROWS;

template <class S> struct SellDev {
  uint32_t rows;                 // one body: its nodes; a batch: every node slot of the system
  uint32_t slices;               // ceil(rows / 32)
  uint32_t positions;            // block positions, a multiple of 32
  uint32_t stride;               // elements of one published vector (>= slices * 32)
  const uint32_t* slice_start;   // [slices + 1]
  const uint32_t* group_slice;   // [positions / 32] slice of each 32-position group
  const uint32_t* col;           // [positions] column node
  uint32_t upper_count;          // block positions with row < column
  uint32_t col_cache;            // column slots per thread kept in shared memory by kPcgSell
  // [upper_count] per block above the diagonal: (position, its transpose's position, first
  // contributor, contributor count | row free << 8 | column free << 9 | body << 10)
  const uint4* urec;
  const uint32_t* centry;        // (element << 4) | (row corner << 2) | column corner
  S* val;                        // [positions / 32][9][32]
  Vec4<S>* vec;                  // [2][stride] published matvec inputs
};

// Block (a, b) of one element's operator, d y_a / d p_b in FP64, where y is
// the element matvec of elementApply.  Corotated law without damping in
// closed form: with gh = R g, sigma(e) = k.x tr(e) I + k.y e - k.z (n : e) n
// and e = sym(p_b gh_b^T),
//   B_ij = k.x gh_a,i gh_b,j + k.y (delta_ij gh_a.gh_b + gh_b,i gh_a,j) / 2
//          - k.z (n gh_a)_i (n gh_b)_j.
// Otherwise the columns are the element operator applied to the three unit
// vectors at corner b.
// v_i for a run-time corner index, by selects (no local-memory array).
template <class T>
__device__ __forceinline__ V3<T> pick(const V3<T>& v0, const V3<T>& v1, const V3<T>& v2, const V3<T>& v3, uint32_t i) {
  return i == 0 ? v0 : i == 1 ? v1 : i == 2 ? v2 : v3;
}

template <class S, int LAW, bool TANGENT, bool DAMP>
__device__ __forceinline__ void addElementBlock(const Sys<S>& s, uint32_t e, uint32_t a, uint32_t b,
                                                double (&acc)[9]) {
  const ElementOperator<S> o = loadOperator<S, LAW, TANGENT>(s, e);
  if constexpr (LAW == 0 && !DAMP) {
    const V3<double> ga = cvt<double>(pick(o.g[0], o.g[1], o.g[2], o.g[3], a)),
                     gb = cvt<double>(pick(o.g[0], o.g[1], o.g[2], o.g[3], b));
    const double kx = double(o.k.x), hy = 0.5 * double(o.k.y);
    const double gg = hy * dot(ga, gb);
    V3<double> na = {0, 0, 0}, nb = {0, 0, 0};
    if (TANGENT) {
      const Sym<double> n = {double(o.n.xx), double(o.n.yy), double(o.n.zz),
                             double(o.n.xy), double(o.n.xz), double(o.n.yz)};
      const double kz = double(o.k.z);
      na = kz * symMul(n, ga);
      nb = symMul(n, gb);
    }
    const double A[3] = {ga.x, ga.y, ga.z}, Bv[3] = {gb.x, gb.y, gb.z};
    const double NA[3] = {na.x, na.y, na.z}, NB[3] = {nb.x, nb.y, nb.z};
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j)
        acc[3 * i + j] += kx * A[i] * Bv[j] + hy * Bv[i] * A[j] + (i == j ? gg : 0.0) - NA[i] * NB[j];
  } else {
#pragma unroll 1
    for (int j = 0; j < 3; ++j) {
      const V3<S> unit = {S(j == 0), S(j == 1), S(j == 2)}, zero = {0, 0, 0};
      V3<S> p[4], y[4];
#pragma unroll
      for (uint32_t c = 0; c < 4; ++c) p[c] = c == b ? unit : zero;
      applyOperator<S, LAW, TANGENT>(o, p, y);
      if (DAMP && LAW == 0) dampingProduct(s, e, o.g, p, y);
      const V3<S> ya = pick(y[0], y[1], y[2], y[3], a);
      acc[j] += double(ya.x);
      acc[3 + j] += double(ya.y);
      acc[6 + j] += double(ya.z);
    }
  }
}

// One thread per block (r, c) with r < c: the sum over its contributors
// (ascending element) is block (r, c), and its transpose is block (c, r),
// since every element block satisfies B_ab = B_ba^T.  A block in an anchored
// row is zero (its transpose, in a free row, is not).  Diagonal blocks are
// written by kNodeAssemble, whose diagonal block of a node (the sum of the
// element pass's corner blocks plus (1 - alpha_m) m I, before its inversion
// into the preconditioner) is this operator's.  Padding positions are zero
// from the build and are never written.
template <class S, int LAW, bool TANGENT, bool DAMP>
__global__ void __launch_bounds__(TILE, 4) kSellAssemble(Sys<S> s, SellDev<S> g, uint32_t pass) {
  const uint32_t i = blockIdx.x * TILE + threadIdx.x;
  if (i >= g.upper_count) return;
  // one record holds what the block needs, so its first contributor's code is requested
  // together with the body's step flags: two dependent loads before the element records
  const uint4 rec = __ldg(&g.urec[i]);
  const uint32_t pos = rec.x, mpos = rec.y, q0 = rec.z, count = rec.w & 0xffu;
  const bool rowFree = ((rec.w >> 8) & 1u) != 0u, colFree = ((rec.w >> 9) & 1u) != 0u;
  const uint32_t body = rec.w >> 10;  // a block's two nodes share a body
  const uint32_t first = count ? __ldg(&g.centry[q0]) : 0u;
  if (!bodyActive(s, body, pass)) return;
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (rowFree || colFree) {
    for (uint32_t q = 0; q < count; ++q) {
      const uint32_t code = q ? __ldg(&g.centry[q0 + q]) : first;
      addElementBlock<S, LAW, TANGENT, DAMP>(s, code >> 4, (code >> 2) & 3u, code & 3u, acc);
    }
  }
  S* v = g.val + size_t(pos >> 5) * 9 * SELL_ROWS + (pos & 31u);
#pragma unroll
  for (int c = 0; c < 9; ++c) v[c * SELL_ROWS] = rowFree ? S(acc[c]) : S(0);
  if (mpos != pos) {
    S* t = g.val + size_t(mpos >> 5) * 9 * SELL_ROWS + (mpos & 31u);
#pragma unroll
    for (int i3 = 0; i3 < 3; ++i3)
#pragma unroll
      for (int j3 = 0; j3 < 3; ++j3) t[(3 * i3 + j3) * SELL_ROWS] = colFree ? S(acc[3 * j3 + i3]) : S(0);
  }
}

// Column k of the thread's row: shared memory for the first col_cache slots
// (filled once per launch by kPcgSell), global memory beyond.
__device__ __forceinline__ uint32_t sellCol(const uint32_t* cols, uint32_t cache, uint32_t k, const uint32_t* gcol,
                                            uint32_t p) {
  return k < cache ? cols[k * TILE + threadIdx.x] : __ldg(&gcol[p]);
}

// One column slot of the thread's row: acc += block(p) x.
template <class S>
__device__ __forceinline__ void sellSlot(const SellDev<S>& g, uint32_t p, uint32_t lane, Vec4<S> xin,
                                         V3<double>& acc) {
  const S* v = g.val + size_t(p >> 5) * 9 * SELL_ROWS + lane;
  const V3<double> x = cvt<double>(xyz(xin));
  const double b0 = __ldg(v), b1 = __ldg(v + 32), b2 = __ldg(v + 64), b3 = __ldg(v + 96), b4 = __ldg(v + 128),
               b5 = __ldg(v + 160), b6 = __ldg(v + 192), b7 = __ldg(v + 224), b8 = __ldg(v + 256);
  acc.x = fma(b0, x.x, fma(b1, x.y, fma(b2, x.z, acc.x)));
  acc.y = fma(b3, x.x, fma(b4, x.y, fma(b5, x.z, acc.y)));
  acc.z = fma(b6, x.x, fma(b7, x.y, fma(b8, x.z, acc.z)));
}

// y = A in for the thread's row.  Column slots are taken U at a time (4 in
// FP32, 2 in FP64): their input values and block entries are requested
// together; the FMAs run slot by slot in order.  With PREFETCH (columns read
// from global memory, as in the batched kernels) the next group's column
// indices are requested with this group's inputs, so a group costs one round
// trip instead of two; kPcgSell reads its columns from shared memory and
// goes without (the extra registers made it slower).
template <class S, class In, uint32_t U = sizeof(S) == 4 ? 4u : 2u, bool PREFETCH = true>
__device__ __forceinline__ V3<double> sellRowOf(const SellDev<S>& g, uint32_t slice, uint32_t lane, In in,
                                                const uint32_t* cols) {
  V3<double> acc = {0, 0, 0};
  const uint32_t p1 = __ldg(&g.slice_start[slice + 1]);
  uint32_t p = __ldg(&g.slice_start[slice]) + lane, k = 0;
  if constexpr (PREFETCH) {
    uint32_t c[U];
#pragma unroll
    for (uint32_t i = 0; i < U; ++i)
      c[i] = p + i * SELL_ROWS < p1 ? sellCol(cols, g.col_cache, k + i, g.col, p + i * SELL_ROWS) : 0u;
    for (; p + (U - 1) * SELL_ROWS < p1; p += U * SELL_ROWS, k += U) {
      Vec4<S> xin[U];
#pragma unroll
      for (uint32_t i = 0; i < U; ++i) xin[i] = in(c[i]);
      const uint32_t pn = p + U * SELL_ROWS;
#pragma unroll
      for (uint32_t i = 0; i < U; ++i)
        c[i] = pn + i * SELL_ROWS < p1 ? sellCol(cols, g.col_cache, k + U + i, g.col, pn + i * SELL_ROWS) : 0u;
#pragma unroll
      for (uint32_t i = 0; i < U; ++i) sellSlot(g, p + i * SELL_ROWS, lane, xin[i], acc);
    }
    // fewer than U slots remain; their columns are in c already
#pragma unroll
    for (uint32_t i = 0; i + 1 < U; ++i)
      if (p + i * SELL_ROWS < p1) sellSlot(g, p + i * SELL_ROWS, lane, in(c[i]), acc);
  } else {
    for (; p + (U - 1) * SELL_ROWS < p1; p += U * SELL_ROWS, k += U) {
      uint32_t c[U];
#pragma unroll
      for (uint32_t i = 0; i < U; ++i) c[i] = sellCol(cols, g.col_cache, k + i, g.col, p + i * SELL_ROWS);
      Vec4<S> xin[U];
#pragma unroll
      for (uint32_t i = 0; i < U; ++i) xin[i] = in(c[i]);
#pragma unroll
      for (uint32_t i = 0; i < U; ++i) sellSlot(g, p + i * SELL_ROWS, lane, xin[i], acc);
    }
    for (; p < p1; p += SELL_ROWS, ++k) sellSlot(g, p, lane, in(sellCol(cols, g.col_cache, k, g.col, p)), acc);
  }
  return acc;
}
// The matvec input read from a vector written during the launch (L2).
template <class S> struct Ld4cg {
  const Vec4<S>* v;
  __device__ __forceinline__ Vec4<S> operator()(uint32_t c) const { return ld4cg(&v[c]); }
};
template <class S> __device__ __forceinline__ Ld4cg<S> ld4cgOf(const Vec4<S>* v) { return Ld4cg<S>{v}; }
// kPcgSell's row: columns from its shared-memory cache, no prefetch, U slots per round trip.
template <class S, uint32_t U>
__device__ __forceinline__ V3<double> sellRow(const SellDev<S>& g, uint32_t slice, uint32_t lane,
                                              const Vec4<S>* in, const uint32_t* cols) {
  return sellRowOf<S, Ld4cg<S>, U, false>(g, slice, lane, ld4cgOf(in), cols);
}
// Column slots per round trip of the assembled matvec rows (a launch shape
// tl_system_tune_shape may change): kPcgSell's default, then the batched kernels'.
template <class S> __host__ __device__ constexpr uint32_t sellRowGroup() { return sizeof(S) == 4 ? 4u : 2u; }
constexpr uint32_t BATCH_ROW_GROUP = 2u;
constexpr int BATCH_BLOCKS = 4;  // resident blocks per SM the batched kernels are compiled for by default

template <class S> __device__ __forceinline__ V3<double> roundTo(V3<double> v) {
  return cvt<double>(cvt<S>(v));
}

// Pipelined PCG (conjugateGradient, solver.cc:1904-2089, block-Jacobi
// branch; Ghysels-Vanroose arrangement).  With u = P r, w = A u, m = P w,
// n = A m, per iteration:
//   gamma = r.u, delta = w.u                    (reduced at the barrier)
//   beta = gamma / gamma_prev, p.A p = delta - beta gamma / alpha_prev,
//   alpha = gamma / p.A p
//   z = n + beta z, q = m + beta q, s = w + beta s, p = u + beta p,
//   x += alpha p, r -= alpha s, u -= alpha q, w -= alpha z,
// where n = A m is computed while the reduction of gamma, delta, r.r is in
// flight.  In exact arithmetic the iterates are the reference's; the stopping
// test (|r| <= tolerance |rhs| or the iteration cap, checked before each
// update), the breakdown test (p.A p > 0 and r.u > 0) and the iteration
// count are the reference's, and a solve that reaches the cap applies its
// last update without a matvec.  Block partials are added in block order, so
// every block takes the same decisions.  The slices of block b are
// [b slices / G, (b + 1) slices / G), at most 8, one per warp.
template <class S, uint32_t U = sellRowGroup<S>()>
__global__ void __launch_bounds__(TILE, 2) kPcgSell(Sys<S> s, SellDev<S> g, Vec4<S>* X, uint32_t x0zero, uint32_t tangent) {
  const uint32_t G = gridDim.x, lane = threadIdx.x & 31u;
  const uint32_t s0 = uint32_t(uint64_t(blockIdx.x) * g.slices / G);
  const uint32_t s1 = uint32_t(uint64_t(blockIdx.x + 1) * g.slices / G);
  const uint32_t slice = s0 + (threadIdx.x >> 5);
  const bool mine = slice < s1;
  const uint32_t row = slice * SELL_ROWS + lane;
  const bool live = mine && row < g.rows;
  const bool freeRow = live && !s.anch[row];
  const BodyStepDev st = s.step[0];
  extern __shared__ uint32_t tlCols[];  // [col_cache][TILE] the first columns of each thread's row
  // the block partials of each iteration's reduction, fetched while the matvec's inputs are
  // (grids of up to SELL_PART_STAGE_BLOCKS blocks; larger ones read them from L2 after it)
  constexpr unsigned SELL_PART_STAGE_BLOCKS = 320;
  __shared__ __align__(16) double partStage[3 * SELL_PART_STAGE_BLOCKS + 2];
  const bool stagedSums = G <= SELL_PART_STAGE_BLOCKS;
  if (mine) {
    const uint32_t p0 = __ldg(&g.slice_start[slice]) + lane, p1 = __ldg(&g.slice_start[slice + 1]);
    for (uint32_t k = 0, p = p0; k < g.col_cache && p < p1; ++k, p += SELL_ROWS)
      tlCols[k * TILE + threadIdx.x] = __ldg(&g.col[p]);
  }
  __syncthreads();
  // Block partials alternate between two halves of blk_part by reduction
  // parity: with one barrier per iteration, a block may write the next
  // reduction's partials while another still sums the previous one.
  double* const halves[2] = {s.blk_part, s.blk_part + 4 * size_t(G)};
  uint32_t reductions = 0;
  unsigned int bar = 0;
  Sym<S> Ps = {1, 1, 1, 0, 0, 0};  // the row's preconditioner block, widened where used
  const auto precondition = [&](V3<double> v) {
    const Sym<double> P = {double(Ps.xx), double(Ps.yy), double(Ps.zz), double(Ps.xy), double(Ps.xz), double(Ps.yz)};
    return roundTo<S>(symMul(P, v));
  };
  V3<double> x = {0, 0, 0}, r = {0, 0, 0}, rhs = {0, 0, 0};
  if (live) {
    const Vec4<S> q0 = s.pre0[row], q1 = s.pre1[row];
    Ps = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y};
    rhs = cvt<double>(xyz(s.right[row]));
    if (!x0zero) x = cvt<double>(xyz(X[row]));
  }
  uint32_t applications = 0;
  // ---- r = right - A x (anchored rows 0), u = P r, published to vec[1]
  if (!x0zero) {
    const V3<double> ax = mine ? sellRow<S, U>(g, slice, lane, X, tlCols) : V3<double>{0, 0, 0};
    if (freeRow) r = rhs - ax;
    ++applications;
  } else if (freeRow) {
    r = rhs;
  }
  V3<double> u = precondition(r);
  Vec4<S>* vec0 = g.vec;
  Vec4<S>* vec1 = g.vec + g.stride;
  if (mine) vec1[row] = pack(cvt<S>(u));
  if (!countBarrier(s.sync, bar)) return;
  // ---- w = A u, m = P w published to vec[0], first reduction
  V3<double> w = mine ? sellRow<S, U>(g, slice, lane, vec1, tlCols) : V3<double>{0, 0, 0};
  ++applications;
  V3<double> m = precondition(w);
  if (mine) vec0[row] = pack(cvt<S>(m));
  {
    double v[4] = {dot(r, u), dot(w, u), dot(r, r), live ? dot(rhs, rhs) : 0.0};
    blockSum<4>(v);
    if (threadIdx.x == 0)
#pragma unroll
      for (int k = 0; k < 4; ++k) halves[0][k * G + blockIdx.x] = v[k];
  }
  if (!countBarrier(s.sync, bar)) return;
  // n = A m for the first iteration, requested before the block sums so that
  // their round trip overlaps it (unused if the solve stops here)
  V3<double> n = mine ? sellRow<S, U>(g, slice, lane, vec0, tlCols) : V3<double>{0, 0, 0};
  double sums[4];
  sumBlocksAll<4>(halves[0], sums);
  ++reductions;
  double gammaNext = sums[0], delta = sums[1], length = sums[2];
  const double reference = sqrt(sums[3]);
  const double floor = fmax(reference, 1.1754943508222875e-38);  // std::numeric_limits<float>::min()
  const double target = st.tolerance * floor;
  const double startRes = sqrt(length) / floor;
  double gamma = 0.0, alpha = 0.0, beta = 0.0;
  uint32_t taken = 0;
  V3<double> zv = {0, 0, 0}, qv = {0, 0, 0}, sv = {0, 0, 0}, pv = {0, 0, 0};
  for (;;) {
    if (taken >= st.limit || sqrt(length) <= target) break;  // the reference's loop-top test
    const double b = taken ? gammaNext / gamma : 0.0;
    const double curvature = taken ? delta - b * gammaNext / alpha : delta;  // p.A p
    if (!(curvature > 0.0) || !(gammaNext > 0.0)) break;
    beta = b;
    alpha = gammaNext / curvature;
    gamma = gammaNext;
    if (taken + 1 >= st.limit) {  // the last update the cap allows: no matvec after it
      pv = u + beta * pv;
      sv = w + beta * sv;
      x = x + alpha * pv;
      r = r - alpha * sv;
      double* part = halves[reductions & 1u];
      double v[3] = {0.0, 0.0, dot(r, r)};
      blockSum<3>(v);
      if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < 3; ++k) part[k * G + blockIdx.x] = v[k];
      if (!countBarrier(s.sync, bar)) return;
      double fin[3];
      sumBlocksAll<3>(part, fin);
      length = fin[2];
      ++taken;
      break;
    }
    ++applications;  // n = A m of this iteration, computed after the last barrier
    zv = n + beta * zv;
    qv = m + beta * qv;
    sv = w + beta * sv;
    pv = u + beta * pv;
    x = x + alpha * pv;
    r = r - alpha * sv;
    u = u - alpha * qv;
    w = w - alpha * zv;
    m = precondition(w);
    if (mine) ((taken & 1u) ? vec0 : vec1)[row] = pack(cvt<S>(m));
    double* part = halves[reductions & 1u];
    {
      double v[3] = {dot(r, u), dot(w, u), dot(r, r)};
      blockSum<3>(v);
      if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < 3; ++k) part[k * G + blockIdx.x] = v[k];
    }
    if (!countBarrier(s.sync, bar)) return;
    // n = A m for the next iteration (m just published to vec[(taken + 1) & 1]), with the
    // block partials requested first so that both round trips overlap
    if (stagedSums) requestBlockPartials(part, partStage, 3u);
    n = mine ? sellRow<S, U>(g, slice, lane, (taken & 1u) ? vec0 : vec1, tlCols) : V3<double>{0, 0, 0};
    double d[3];
    if (stagedSums) {
      cpAsyncWaitAll();
      __syncthreads();
      sumStagedBlocks<3>(partStage, d);
    } else {
      sumBlocksAll<3>(part, d);
    }
    ++reductions;
    gammaNext = d[0];
    delta = d[1];
    length = d[2];
    ++taken;
  }
  if (live) X[row] = pack(cvt<S>(x));
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
    rep.tangent_iterations += tangent ? taken : 0u;
    rep.worst_rel = fmax(rep.worst_rel, c.rel_res);
    if (rep.pass_solves == 0u) rep.pass_start = c.start_res;
    rep.pass_end = c.rel_res;
    rep.pass_iterations += c.taken;
    rep.pass_solves += 1u;
    s.cgrep[0] = rep;
  }
}

// Persistent PCG over every body of a batched system on the assembled block
// matrix: kPcgBatch's per-body scalars, stopping tests and reports
// (conjugateGradient, solver.cc:1904-2089, block-Jacobi branch), with the
// element matvec and the node gather replaced by the rows of the matrix.
// Per iteration, over node tiles:
//   AB  p = z + beta p_prev and Ap = A p, each neighbour's p formed from its
//       z and p_prev; p.Ap per body -> alpha (last tile of the body)
//   C   x += alpha p, r -= alpha Ap, z = P r; r.z, r.r per body -> beta,
//       stopping test
// with a grid barrier after each.  AB reads the neighbours' previous p while
// writing the new one, so p alternates between two buffers by iteration.
//
// A block's tiles are blockIdx.x + j G (slot j); their bodies and row counts
// are read once per launch into shared memory (tlBatchSlots, 8 bytes per
// slot), and the next live slot's stopping flag and scalar are requested
// while the current tile is worked, so a tile starts without a round trip.
// A body's flag changes within a phase only in its last-arriving tile, after
// every tile of the body has read it.
__device__ __forceinline__ uint32_t nextSlot(const uint32_t* slotBody, uint32_t j, uint32_t slots) {
  while (j < slots && slotBody[j] == ~0u) ++j;
  return j;
}

template <class S, uint32_t U = BATCH_ROW_GROUP, int MINB = BATCH_BLOCKS>
__global__ void __launch_bounds__(TILE, MINB)
    kPcgBatchSell(Sys<S> s, SellDev<S> g, Vec4<S>* X, Vec4<S>* p2, uint32_t pass, uint32_t x0zero, uint32_t tangent) {
  extern __shared__ uint32_t tlBatchSlots[];  // [slots] body (~0u: not stepping), then [slots] rows
  const uint32_t G = gridDim.x, lane = threadIdx.x & 31u;
  g.col_cache = 0;  // no per-launch column cache: a block walks many slices
  const S zero = S(0);
  unsigned int bar = 0;
  const uint32_t slots = blockIdx.x < s.node_tiles ? (s.node_tiles - 1u - blockIdx.x) / G + 1u : 0u;
  uint32_t* const slotBody = tlBatchSlots;
  uint32_t* const slotRows = tlBatchSlots + slots;
  for (uint32_t j = threadIdx.x; j < slots; j += TILE) {
    const uint32_t tile = blockIdx.x + j * G;
    const uint32_t b = s.node_tile_body[tile];
    const bool live = bodyActive(s, b, pass);
    slotBody[j] = live ? b : ~0u;
    slotRows[j] = live ? min(TILE, s.body[b].node_end - tile * TILE) : 0u;
  }
  __syncthreads();
  // ---- init: r = right - A x (anchored rows 0), z = P r, p_prev = 0
  for (uint32_t j = nextSlot(slotBody, 0u, slots); j < slots; j = nextSlot(slotBody, j + 1u, slots)) {
    const uint32_t b = slotBody[j], tile = blockIdx.x + j * G;
    const BodyDev bd = s.body[b];
    const uint32_t n = tile * TILE + threadIdx.x;
    double sums[3] = {0.0, 0.0, 0.0};
    if (threadIdx.x < slotRows[j]) {
      const Vec4<S> rhs = s.right[n];
      V3<S> r = {zero, zero, zero};
      if (!s.anch[n]) {
        V3<double> ax = {0, 0, 0};
        if (!x0zero)
          ax = sellRowOf<S, decltype(ld4cgOf(X)), U>(g, n >> 5, lane, ld4cgOf(X), static_cast<const uint32_t*>(nullptr));
        r = cvt<S>(cvt<double>(xyz(rhs)) - ax);
      }
      const Vec4<S> q0 = s.pre0[n], q1 = s.pre1[n];
      const Sym<S> P = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y};
      const V3<S> z = symMul(P, r);
      s.r[n] = pack(r);
      s.z[n] = pack(z);
      s.p[n] = Vec4<S>{zero, zero, zero, zero};
      if (x0zero) X[n] = Vec4<S>{zero, zero, zero, zero};  // X is multiplied only when !x0zero
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
  for (uint32_t it = 0;; ++it) {
    // uniform: the count changes only in C, whose barrier every block has passed
    if (*(volatile int*)&s.sync->active <= 0) break;
    const Vec4<S>* pprev = (it & 1u) ? p2 : s.p;
    Vec4<S>* pnew = (it & 1u) ? s.p : p2;
    // ---- AB
    uint32_t j = nextSlot(slotBody, 0u, slots), done = 1u;
    double blendNow = 0.0;
    if (j < slots) {
      done = __ldcg(&s.cg[slotBody[j]].done);
      blendNow = __ldcg(&s.cg[slotBody[j]].blend);
    }
    while (j < slots) {
      const uint32_t b = slotBody[j], tile = blockIdx.x + j * G, rows = slotRows[j];
      const uint32_t jn = nextSlot(slotBody, j + 1u, slots);
      uint32_t doneNext = 1u;
      double blendNext = 0.0;
      if (jn < slots) {
        doneNext = __ldcg(&s.cg[slotBody[jn]].done);
        blendNext = __ldcg(&s.cg[slotBody[jn]].blend);
      }
      if (!done) {
        const BodyDev bd = s.body[b];
        const uint32_t n = tile * TILE + threadIdx.x;
        double sums[1] = {0.0};
        if (threadIdx.x < rows) {
          const S blend = S(blendNow);
          const auto pOf = [&](uint32_t c) {
            return pack(fmaV(blend, xyz(ld4cg(&pprev[c])), xyz(ld4cg(&s.z[c]))));
          };
          const V3<S> pn = xyz(pOf(n));
          pnew[n] = pack(pn);
          V3<S> apn = {zero, zero, zero};
          if (!s.anch[n])
            apn = cvt<S>(sellRowOf<S, decltype(pOf), U>(g, n >> 5, lane, pOf, static_cast<const uint32_t*>(nullptr)));
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
            // a breakdown stops the body without an update; it is retired in C,
            // so that no block changes the active count before this barrier
            s.cg[b].pad0 = (!(curvature > 0.0) || !(squared > 0.0)) ? 1u : 0u;
            s.cg[b].stride = s.cg[b].pad0 ? 0.0 : squared / curvature;
            __threadfence();
          }
        }
      }
      j = jn;
      done = doneNext;
      blendNow = blendNext;
    }
    if (!countBarrier(s.sync, bar)) return;
    // ---- C
    j = nextSlot(slotBody, 0u, slots);
    done = 1u;
    double strideNow = 0.0;
    uint32_t brokenNow = 0u;
    if (j < slots) {
      done = __ldcg(&s.cg[slotBody[j]].done);
      strideNow = __ldcg(&s.cg[slotBody[j]].stride);
      brokenNow = __ldcg(&s.cg[slotBody[j]].pad0);
    }
    while (j < slots) {
      const uint32_t b = slotBody[j], tile = blockIdx.x + j * G, rows = slotRows[j];
      const uint32_t jn = nextSlot(slotBody, j + 1u, slots);
      uint32_t doneNext = 1u, brokenNext = 0u;
      double strideNext = 0.0;
      if (jn < slots) {
        doneNext = __ldcg(&s.cg[slotBody[jn]].done);
        strideNext = __ldcg(&s.cg[slotBody[jn]].stride);
        brokenNext = __ldcg(&s.cg[slotBody[jn]].pad0);
      }
      if (!done) {
        const BodyDev bd = s.body[b];
        const uint32_t n = tile * TILE + threadIdx.x;
        double sums[2] = {0.0, 0.0};
        if (threadIdx.x < rows && !brokenNow) {
          const S stride = S(strideNow);
          const V3<S> pn = xyz(ld4cg(&pnew[n]));
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
            if (c.pad0) {  // broke down in AB: no update, the last residual stands
              c.done = 1u;
            } else {
              c.blend = tot[0] / c.squared;
              c.squared = tot[0];
              c.length = tot[1];
              c.taken += 1u;
              c.done = (sqrt(c.length) <= c.target || c.taken >= s.step[b].limit) ? 1u : 0u;
            }
            s.cg[b] = c;
            __threadfence();
            if (c.done) atomicSub(&s.sync->active, 1);
          }
        }
      }
      j = jn;
      done = doneNext;
      strideNow = strideNext;
      brokenNow = brokenNext;
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

// The batched PCG of kPcgBatchSell in kPcgSell's pipelined arrangement
// (Ghysels-Vanroose): one grid barrier per iteration.  Each body keeps the
// recurrences of kPcgSell in FP64, as kPcgSell keeps them in registers, here
// stored per node (x, r, u = P r, w = A u and z, q, s, p: eight planes of
// Vec4<double>), and m = P w, rounded to S, is published for the next matvec
// n = A m, in two buffers that alternate by phase; X follows x in S.  Per phase, over the block's live tiles:
//   n = A m; z = n + beta z, q = m + beta q, s = w + beta s, p = u + beta p,
//   x += alpha p, r -= alpha s, u -= alpha q, w -= alpha z, m = P w;
//   r.u, w.u, r.r per tile
// and the last tile of each body to arrive sums the body's partials and takes
// the next step of the body's control, as kPcgSell's loop top does: the
// stopping test (|r| <= tolerance |rhs| or the cap), the breakdown test
// (p.A p > 0 and r.u > 0), alpha and beta, and whether the next update is the
// last one the cap allows (p, s, x and r only, no matvec).  A body's flags and
// scalars (cg[b]: squared = gamma, stride = alpha, blend = beta, pad0 = the
// kind of its next update, pad1 = operator applications, done = 1 + the phase
// it stopped in) are read by its tiles after the barrier.
//
// The active count is read at the top of every phase by every block, while
// last tiles of that same phase may already retire bodies, so it is kept in
// two copies: phase k reads copy k & 1 and retires bodies from that copy
// only; a body retired in phase k leaves copy (k + 1) & 1 in phase k + 1,
// through the block that holds its first tile.
constexpr uint32_t PIPE_FULL = 0u;  // kinds of a body's next update
constexpr uint32_t PIPE_LAST = 1u;

// kPcgSell's loop top for one body (thread 0 of its last tile): given the
// sums gamma' = r.u, delta = w.u and |r|^2 of the current iterate, either stop
// or set alpha, beta and the kind of the next update.
__device__ __forceinline__ void pipeDecide(CgBodyDev& c, double gammaNext, double delta, uint32_t limit,
                                           uint32_t phase) {
  if (c.taken >= limit || sqrt(c.length) <= c.target) {
    c.done = phase + 1u;
    return;
  }
  const double b = c.taken ? gammaNext / c.squared : 0.0;
  const double curvature = c.taken ? delta - b * gammaNext / c.stride : delta;  // p.A p
  if (!(curvature > 0.0) || !(gammaNext > 0.0)) {
    c.done = phase + 1u;
    return;
  }
  c.blend = b;
  c.stride = gammaNext / curvature;
  c.squared = gammaNext;
  c.pad0 = c.taken + 1u >= limit ? PIPE_LAST : PIPE_FULL;
  if (c.pad0 == PIPE_FULL) c.pad1 += 1u;  // the matvec n = A m of the update
}

template <class S, uint32_t U = BATCH_ROW_GROUP, int MINB = BATCH_BLOCKS>
__global__ void __launch_bounds__(TILE, MINB)
    kPcgBatchSellPipe(Sys<S> s, SellDev<S> g, Vec4<S>* X, Vec4<double>* state, uint32_t pass, uint32_t x0zero,
                      uint32_t tangent) {
  extern __shared__ uint32_t tlBatchSlots[];  // [slots] body (~0u: not stepping), then [slots] rows
  const uint32_t G = gridDim.x, lane = threadIdx.x & 31u;
  g.col_cache = 0;
  unsigned int bar = 0;
  const uint32_t slots = blockIdx.x < s.node_tiles ? (s.node_tiles - 1u - blockIdx.x) / G + 1u : 0u;
  uint32_t* const slotBody = tlBatchSlots;
  uint32_t* const slotRows = tlBatchSlots + slots;  // rows, | 0x80000000 on the first tile of its body
  for (uint32_t j = threadIdx.x; j < slots; j += TILE) {
    const uint32_t tile = blockIdx.x + j * G;
    const uint32_t b = s.node_tile_body[tile];
    const bool live = bodyActive(s, b, pass);
    slotBody[j] = live ? b : ~0u;
    const BodyDev bd = s.body[b];
    slotRows[j] = live ? (min(TILE, bd.node_end - tile * TILE) | (tile == bd.node_tile_begin ? 0x80000000u : 0u)) : 0u;
  }
  __syncthreads();
  Vec4<S>* const vecA = g.vec;             // m of even phases (and of phase 0)
  Vec4<S>* const vecB = g.vec + g.stride;  // u of the start, then m of odd phases
  // the FP64 recurrences, [8][Vp]: x, r, u, w, z, q, s, p (in an FP64 system x is X itself)
  constexpr bool wide = std::is_same_v<S, double>;
  Vec4<double>* const xd = wide ? reinterpret_cast<Vec4<double>*>(X) : state;
  Vec4<double>* const rd = state + size_t(s.Vp);
  Vec4<double>* const u = state + 2 * size_t(s.Vp);
  Vec4<double>* const w = state + 3 * size_t(s.Vp);
  Vec4<double>* const zbuf = state + 4 * size_t(s.Vp);
  Vec4<double>* const qbuf = state + 5 * size_t(s.Vp);
  Vec4<double>* const sv = state + 6 * size_t(s.Vp);
  Vec4<double>* const p = state + 7 * size_t(s.Vp);
  const Vec4<S> zero4 = {S(0), S(0), S(0), S(0)};
  const Vec4<double> zero4d = {0.0, 0.0, 0.0, 0.0};
  const auto get = [](const Vec4<double>* v, uint32_t n) { return xyz(v[n]); };
  const auto put = [](Vec4<double>* v, uint32_t n, V3<double> a) { v[n] = pack(a); };
  const auto precondition = [&](uint32_t n, V3<double> v) {
    const Vec4<S> q0 = s.pre0[n], q1 = s.pre1[n];
    const Sym<double> P = {double(q0.x), double(q0.y), double(q0.z), double(q0.w), double(q1.x), double(q1.y)};
    return roundTo<S>(symMul(P, v));
  };
  // ---- start: r = right - A x (anchored rows 0), u = P r published; the recurrences start at 0
  for (uint32_t j = nextSlot(slotBody, 0u, slots); j < slots; j = nextSlot(slotBody, j + 1u, slots)) {
    const uint32_t tile = blockIdx.x + j * G;
    const uint32_t n = tile * TILE + threadIdx.x;
    if (threadIdx.x >= (slotRows[j] & 0x7fffffffu)) continue;
    V3<double> r = {0, 0, 0};
    if (!s.anch[n]) {
      V3<double> ax = {0, 0, 0};
      if (!x0zero)
        ax = sellRowOf<S, decltype(ld4cgOf(X)), U>(g, n >> 5, lane, ld4cgOf(X), static_cast<const uint32_t*>(nullptr));
      r = cvt<double>(xyz(s.right[n])) - ax;
    }
    const V3<double> uu = precondition(n, r);
    put(rd, n, r);
    put(u, n, uu);
    vecB[n] = pack(cvt<S>(uu));
    if (x0zero) X[n] = zero4;
    if (!wide) xd[n] = x0zero ? zero4d : pack(cvt<double>(xyz(X[n])));
    zbuf[n] = zero4d;
    qbuf[n] = zero4d;
    sv[n] = zero4d;
    p[n] = zero4d;
  }
  if (!countBarrier(s.sync, bar)) return;
  // ---- phase 0: w = A u, m = P w published; r.u, w.u, r.r, rhs.rhs per body -> the first decision
  for (uint32_t j = nextSlot(slotBody, 0u, slots); j < slots; j = nextSlot(slotBody, j + 1u, slots)) {
    const uint32_t b = slotBody[j], tile = blockIdx.x + j * G;
    const uint32_t n = tile * TILE + threadIdx.x;
    double sums[4] = {0.0, 0.0, 0.0, 0.0};
    if (threadIdx.x < (slotRows[j] & 0x7fffffffu)) {
      V3<double> ww = {0, 0, 0};
      if (!s.anch[n])
        ww = sellRowOf<S, decltype(ld4cgOf(vecB)), U>(g, n >> 5, lane, ld4cgOf(vecB), static_cast<const uint32_t*>(nullptr));
      const V3<double> m = precondition(n, ww);
      put(w, n, ww);
      vecA[n] = pack(cvt<S>(m));
      const V3<double> r = get(rd, n), uu = get(u, n);
      const V3<double> rhs = cvt<double>(xyz(s.right[n]));
      sums[0] = dot(r, uu);
      sums[1] = dot(ww, uu);
      sums[2] = dot(r, r);
      sums[3] = dot(rhs, rhs);
    }
    blockSum<4>(sums);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < 4; ++k) s.part[size_t(tile) * 4 + k] = sums[k];
    }
    const BodyDev bd = s.body[b];
    if (lastTileOfBody(&s.counter[b], bd.node_tile_end - bd.node_tile_begin)) {
      double tot[4];
      sumTiles<4>(s.part, bd.node_tile_begin, bd.node_tile_end, tot);
      if (threadIdx.x == 0) {
        CgBodyDev c;
        const double reference = sqrt(tot[3]);
        c.floor = fmax(reference, 1.1754943508222875e-38);  // std::numeric_limits<float>::min()
        c.target = s.step[b].tolerance * c.floor;
        c.length = tot[2];
        c.start_res = sqrt(tot[2]) / c.floor;
        c.rel_res = c.start_res;
        c.squared = 0.0;
        c.stride = 0.0;
        c.blend = 0.0;
        c.taken = 0;
        c.done = 0;
        c.pad0 = PIPE_FULL;
        c.pad1 = (x0zero ? 0u : 1u) + 1u;  // r = right - A x and w = A u
        pipeDecide(c, tot[0], tot[1], s.step[b].limit, 0u);
        s.cg[b] = c;
        __threadfence();
        if (c.done) atomicSub(&s.sync->active, 1);
      }
    }
  }
  if (!countBarrier(s.sync, bar)) return;
  for (uint32_t phase = 1;; ++phase) {
    // the count of phase - 1's copy: retirements of this phase go to the other copy
    if (*(volatile int*)(((phase - 1u) & 1u) ? &s.sync->active_odd : &s.sync->active) <= 0) break;
    int* const retire = (phase & 1u) ? &s.sync->active_odd : &s.sync->active;
    const Vec4<S>* const mcur = (phase & 1u) ? vecA : vecB;
    Vec4<S>* const mnext = (phase & 1u) ? vecB : vecA;
    uint32_t j = nextSlot(slotBody, 0u, slots);
    CgBodyDev cNow = {};
    if (j < slots) cNow = loadCg(&s.cg[slotBody[j]]);
    while (j < slots) {
      const uint32_t b = slotBody[j], tile = blockIdx.x + j * G, rowsWord = slotRows[j];
      const uint32_t jn = nextSlot(slotBody, j + 1u, slots);
      CgBodyDev cNext = {};
      if (jn < slots) cNext = loadCg(&s.cg[slotBody[jn]]);
      if (cNow.done) {
        // retired in the previous phase: leave this phase's copy of the count too
        if (cNow.done == phase && (rowsWord & 0x80000000u) && threadIdx.x == 0) atomicSub(retire, 1);
      } else {
        const uint32_t n = tile * TILE + threadIdx.x;
        const double alpha = cNow.stride, beta = cNow.blend;
        double sums[3] = {0.0, 0.0, 0.0};
        if (threadIdx.x < (rowsWord & 0x7fffffffu)) {
          const bool full = cNow.pad0 == PIPE_FULL;
          // the matvec first: its round trips are the phase's latency
          V3<double> nn = {0, 0, 0};
          if (full && !s.anch[n])
            nn = sellRowOf<S, decltype(ld4cgOf(mcur)), U>(g, n >> 5, lane, ld4cgOf(mcur),
                                                          static_cast<const uint32_t*>(nullptr));
          const V3<double> uu = get(u, n), ww = get(w, n);
          const V3<double> pp = uu + beta * get(p, n);
          const V3<double> ss = ww + beta * get(sv, n);
          const V3<double> x = get(xd, n) + alpha * pp;
          const V3<double> r = get(rd, n) - alpha * ss;
          put(p, n, pp);
          put(sv, n, ss);
          put(xd, n, x);
          if (!wide) X[n] = pack(cvt<S>(x));
          put(rd, n, r);
          if (full) {
            const V3<double> m = cvt<double>(xyz(ld4cg(&mcur[n])));
            const V3<double> zz = nn + beta * get(zbuf, n);
            const V3<double> qq = m + beta * get(qbuf, n);
            const V3<double> u2 = uu - alpha * qq;
            const V3<double> w2 = ww - alpha * zz;
            put(zbuf, n, zz);
            put(qbuf, n, qq);
            put(u, n, u2);
            put(w, n, w2);
            mnext[n] = pack(cvt<S>(precondition(n, w2)));
            sums[0] = dot(r, u2);
            sums[1] = dot(w2, u2);
          }
          sums[2] = dot(r, r);
        }
        blockSum<3>(sums);
        if (threadIdx.x == 0) {
#pragma unroll
          for (int k = 0; k < 3; ++k) s.part[size_t(tile) * 4 + k] = sums[k];
        }
        const BodyDev bd = s.body[b];
        if (lastTileOfBody(&s.counter[b], bd.node_tile_end - bd.node_tile_begin)) {
          double tot[3];
          sumTiles<3>(s.part, bd.node_tile_begin, bd.node_tile_end, tot);
          if (threadIdx.x == 0) {
            CgBodyDev c = loadCg(&s.cg[b]);
            c.length = tot[2];
            c.taken += 1u;
            if (c.pad0 == PIPE_LAST)
              c.done = phase + 1u;
            else
              pipeDecide(c, tot[0], tot[1], s.step[b].limit, phase);
            s.cg[b] = c;
            __threadfence();
            if (c.done) atomicSub(retire, 1);
          }
        }
      }
      j = jn;
      cNow = cNext;
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
      s.cg[b].done = 1u;
      CgReportDev rep = s.cgrep[b];
      rep.iterations += c.taken;
      rep.capped += (c.taken == s.step[b].limit && residual > c.target) ? 1u : 0u;
      rep.applications += c.pad1;
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

}  // namespace tl
