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
//   kPcgBatchSell  the batched PCG of kPcgBatch on this matrix, for batches
//                  and for single bodies with more rows than kPcgSell's grid
//                  has threads;
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
  const uint32_t* upper;         // [upper_count] those positions
  const uint32_t* mirror;        // [upper_count] position of the transposed block
  const uint32_t* cstart;        // [positions + 1] contributor range of each position
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
  const uint32_t pos = g.upper[i], mpos = g.mirror[i];
  const uint32_t row = g.group_slice[pos >> 5] * SELL_ROWS + (pos & 31u), col = g.col[pos];
  const uint32_t body = s.node_tile_body[row / TILE];  // a block's two nodes share a body
  if (!bodyActive(s, body, pass)) return;
  const bool rowFree = !s.anch[row], colFree = !s.anch[col];
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (rowFree || colFree) {
    const uint32_t q1 = g.cstart[pos + 1];
    for (uint32_t q = g.cstart[pos]; q < q1; ++q) {
      const uint32_t code = __ldg(&g.centry[q]);
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
// together; the FMAs run slot by slot in order.
template <class S, class In, uint32_t U = sizeof(S) == 4 ? 4u : 2u>
__device__ __forceinline__ V3<double> sellRowOf(const SellDev<S>& g, uint32_t slice, uint32_t lane, In in,
                                                const uint32_t* cols) {
  V3<double> acc = {0, 0, 0};
  const uint32_t p1 = __ldg(&g.slice_start[slice + 1]);
  uint32_t p = __ldg(&g.slice_start[slice]) + lane, k = 0;
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
  return acc;
}
// The matvec input read from a vector written during the launch (L2).
template <class S> struct Ld4cg {
  const Vec4<S>* v;
  __device__ __forceinline__ Vec4<S> operator()(uint32_t c) const { return ld4cg(&v[c]); }
};
template <class S> __device__ __forceinline__ Ld4cg<S> ld4cgOf(const Vec4<S>* v) { return Ld4cg<S>{v}; }
template <class S>
__device__ __forceinline__ V3<double> sellRow(const SellDev<S>& g, uint32_t slice, uint32_t lane,
                                              const Vec4<S>* in, const uint32_t* cols) {
  return sellRowOf(g, slice, lane, ld4cgOf(in), cols);
}

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
template <class S>
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
    const V3<double> ax = mine ? sellRow(g, slice, lane, X, tlCols) : V3<double>{0, 0, 0};
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
  V3<double> w = mine ? sellRow(g, slice, lane, vec1, tlCols) : V3<double>{0, 0, 0};
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
  V3<double> n = mine ? sellRow(g, slice, lane, vec0, tlCols) : V3<double>{0, 0, 0};
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
    // n = A m for the next iteration (m just published to vec[(taken + 1) & 1])
    n = mine ? sellRow(g, slice, lane, (taken & 1u) ? vec0 : vec1, tlCols) : V3<double>{0, 0, 0};
    double d[3];
    sumBlocksAll<3>(part, d);
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
template <class S>
__global__ void __launch_bounds__(TILE, 4)
    kPcgBatchSell(Sys<S> s, SellDev<S> g, Vec4<S>* X, Vec4<S>* p2, uint32_t pass, uint32_t x0zero, uint32_t tangent) {
  const uint32_t G = gridDim.x, lane = threadIdx.x & 31u;
  g.col_cache = 0;  // no per-launch column cache: a block walks many slices
  const S zero = S(0);
  unsigned int bar = 0;
  Vec4<S>* const pbuf[2] = {s.p, p2};
  // ---- init: r = right - A x (anchored rows 0), z = P r, p_prev = 0
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
          ax = sellRowOf<S, decltype(ld4cgOf(X)), 2u>(g, n >> 5, lane, ld4cgOf(X), static_cast<const uint32_t*>(nullptr));
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
    if (*(volatile int*)&s.sync->active <= 0) break;  // uniform: no block decrements between here and barrier AB
    const Vec4<S>* pprev = pbuf[it & 1u];
    Vec4<S>* pnew = pbuf[(it + 1u) & 1u];
    // ---- AB
    for (uint32_t tile = blockIdx.x; tile < s.node_tiles; tile += G) {
      const uint32_t b = s.node_tile_body[tile];
      if (!bodyActive(s, b, pass) || __ldcg(&s.cg[b].done)) continue;
      const BodyDev bd = s.body[b];
      const uint32_t n = tile * TILE + threadIdx.x;
      double sums[1] = {0.0};
      if (n < bd.node_end) {
        const S blend = S(__ldcg(&s.cg[b].blend));
        const auto pOf = [&](uint32_t c) {
          return pack(fmaV(blend, xyz(ld4cg(&pprev[c])), xyz(ld4cg(&s.z[c]))));
        };
        const V3<S> pn = xyz(pOf(n));
        pnew[n] = pack(pn);
        V3<S> apn = {zero, zero, zero};
        if (!s.anch[n])
          apn = cvt<S>(sellRowOf<S, decltype(pOf), 2u>(g, n >> 5, lane, pOf, static_cast<const uint32_t*>(nullptr)));
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
