// tl_factor_host.h -- the block Cholesky factor of a solver state, made on the host.
//
// The system of SystemFactor (factor.cc:318-460) in 3x3 node blocks:
//   A_nn = (1 - alpha_m) m_n I + sum_e h^2 R K_nn R^T, A_nm = sum_e h^2 R K_nm R^T
// over free nodes, anchored nodes carrying the identity and no coupling.
// The reference factors it with Eigen's SimplicialLLT under an AMD ordering
// (factor.cc:302-314); here a nested dissection of the node graph by
// coordinate bisection orders it, the elimination tree and row patterns are
// found once per mesh (analyze), and the numeric factor is an up-looking
// block Cholesky, row by row (factor).  L L^T equals P A P^T to rounding
// whatever the order, so the applied inverse is the reference's.
#pragma once

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <thread>
#include <vector>

#include "tl_math.cuh"

namespace tl {

// factor.cc:49-88 preciseTetBlocks: the 16 blocks step^2 R K R^T in FP64,
// row-major, with Dm and V recomputed from the rest positions (q: the
// tet's nodes, R row-major; preciseLame, factor.cc:21-30).
inline void factorTetBlocks(const double* rest, const uint32_t* q, double youngs, double poisson, const double* R,
                            double step, double* out) {
  double m[3][3];  // columns: the edges from node 0
  for (int k = 0; k < 3; ++k)
    for (int r = 0; r < 3; ++r) m[r][k] = rest[3 * size_t(q[k + 1]) + r] - rest[3 * size_t(q[0]) + r];
  const double c00 = m[1][1] * m[2][2] - m[1][2] * m[2][1], c01 = m[1][2] * m[2][0] - m[1][0] * m[2][2],
               c02 = m[1][0] * m[2][1] - m[1][1] * m[2][0];
  const double det = m[0][0] * c00 + m[0][1] * c01 + m[0][2] * c02;
  const double volume = det / 6.0, inv = 1.0 / det;
  // rows of m^-1 = the gradients of nodes 1..3 (adjugate / determinant)
  double g[4][3];
  g[1][0] = c00 * inv;
  g[2][0] = c01 * inv;
  g[3][0] = c02 * inv;
  g[1][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * inv;
  g[2][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * inv;
  g[3][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * inv;
  g[1][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * inv;
  g[2][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * inv;
  g[3][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * inv;
  for (int r = 0; r < 3; ++r) g[0][r] = -(g[1][r] + g[2][r] + g[3][r]);
  const double nu = std::clamp(poisson, 0.0, 0.49);
  const double lambda = youngs * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), mu = youngs / (2.0 * (1.0 + nu));
  const double scale = step * step;
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      const double gab = g[a][0] * g[b][0] + g[a][1] * g[b][1] + g[a][2] * g[b][2];
      double k[3][3], t[3][3];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          k[i][j] = volume * (lambda * g[a][i] * g[b][j] + mu * g[b][i] * g[a][j] + (i == j ? mu * gab : 0.0));
      for (int i = 0; i < 3; ++i)  // t = R k
        for (int j = 0; j < 3; ++j) t[i][j] = R[3 * i] * k[0][j] + R[3 * i + 1] * k[1][j] + R[3 * i + 2] * k[2][j];
      double* o = out + 9 * (4 * a + b);
      for (int i = 0; i < 3; ++i)  // o = step^2 t R^T
        for (int j = 0; j < 3; ++j)
          o[3 * i + j] = scale * (t[i][0] * R[3 * j] + t[i][1] * R[3 * j + 1] + t[i][2] * R[3 * j + 2]);
    }
}

// factor.cc:274-298, 780-853 dampingBlocks: the 16 blocks of Pi R K R^T Pi,
// Pi the removal of the rigid motion fitted to the corners x (rigidFit,
// factor.cc:780-818: mean translation and the spin I^-1 sum a x v about the
// centroid, I pseudo-inverted when nearly singular), K from Dm^-1 and V
// (tetStiffness, material.cc:209-234), in FP64, row-major.
inline void factorDampingBlocks(const double* x, const double* R, const double* Dm, double volume, double youngs,
                                double poisson, double* out) {
  double centre[3] = {0, 0, 0}, arm[4][3], I[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 3; ++r) centre[r] += x[3 * c + r];
  for (int r = 0; r < 3; ++r) centre[r] *= 0.25;
  for (int c = 0; c < 4; ++c) {
    for (int r = 0; r < 3; ++r) arm[c][r] = x[3 * c + r] - centre[r];
    const double aa = arm[c][0] * arm[c][0] + arm[c][1] * arm[c][1] + arm[c][2] * arm[c][2];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) I[i][j] += (i == j ? aa : 0.0) - arm[c][i] * arm[c][j];
  }
  const double third = (I[0][0] + I[1][1] + I[2][2]) / 3.0;
  M3<double> m;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) m.m[i][j] = I[i][j];
  double inv[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  const double det = det3(m);
  if (det > 1.0e-6 * third * third * third) {
    const M3<double> cf = cofactor(m);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) inv[i][j] = cf.m[j][i] / det;
  } else {
    double a[3][3], v[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) a[i][j] = I[i][j];
    jacobiEigen3(a, v);
    for (int k = 0; k < 3; ++k) {
      if (!(a[k][k] > 1.0e-6 * third)) continue;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) inv[i][j] += v[i][k] * v[j][k] / a[k][k];
    }
  }
  auto removeRigid = [&](double v[4][3]) {
    double mean[3] = {0, 0, 0}, moment[3] = {0, 0, 0}, spin[3];
    for (int c = 0; c < 4; ++c)
      for (int r = 0; r < 3; ++r) {
        mean[r] += v[c][r];
        moment[r] += arm[c][(r + 1) % 3] * v[c][(r + 2) % 3] - arm[c][(r + 2) % 3] * v[c][(r + 1) % 3];
      }
    for (int r = 0; r < 3; ++r) {
      mean[r] *= 0.25;
      spin[r] = inv[r][0] * moment[0] + inv[r][1] * moment[1] + inv[r][2] * moment[2];
    }
    for (int c = 0; c < 4; ++c)
      for (int r = 0; r < 3; ++r)
        v[c][r] -= mean[r] + spin[(r + 1) % 3] * arm[c][(r + 2) % 3] - spin[(r + 2) % 3] * arm[c][(r + 1) % 3];
  };
  double g[4][3];
  for (int k = 0; k < 3; ++k)
    for (int r = 0; r < 3; ++r) g[k + 1][r] = Dm[3 * k + r];
  for (int r = 0; r < 3; ++r) g[0][r] = -(g[1][r] + g[2][r] + g[3][r]);
  const double nu = std::clamp(poisson, 0.0, 0.49);
  const double lambda = youngs * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), mu = youngs / (2.0 * (1.0 + nu));
  for (int corner = 0; corner < 4; ++corner)
    for (int axis = 0; axis < 3; ++axis) {
      double v[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, un[4][3], y[4][3];
      v[corner][axis] = 1.0;
      removeRigid(v);
      for (int c = 0; c < 4; ++c)  // R^T v
        for (int r = 0; r < 3; ++r) un[c][r] = R[r] * v[c][0] + R[3 + r] * v[c][1] + R[6 + r] * v[c][2];
      for (int row = 0; row < 4; ++row) {
        double sum[3] = {0, 0, 0};
        for (int col = 0; col < 4; ++col) {
          const double gab = g[row][0] * g[col][0] + g[row][1] * g[col][1] + g[row][2] * g[col][2];
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
              sum[i] += volume * (lambda * g[row][i] * g[col][j] + mu * g[col][i] * g[row][j] + (i == j ? mu * gab : 0.0)) *
                        un[col][j];
        }
        for (int r = 0; r < 3; ++r) y[row][r] = R[3 * r] * sum[0] + R[3 * r + 1] * sum[1] + R[3 * r + 2] * sum[2];
      }
      removeRigid(y);
      for (int row = 0; row < 4; ++row)
        for (int r = 0; r < 3; ++r) out[9 * (4 * row + corner) + 3 * r + axis] = y[row][r];
    }
}


struct BlockFactor {
  uint32_t nodes = 0;
  bool analyzed = false, ready = false;
  uint64_t systemNonZeros = 0;  // stored entries of the full scalar system, as the reference counts them
  std::vector<uint32_t> perm, iperm;          // factor order -> node, node -> factor order
  std::vector<uint32_t> rowStart, rowCol;     // strictly lower blocks of L by rows, columns ascending
  std::vector<uint32_t> colStart, colRow;     // the same blocks by columns, rows ascending
  std::vector<double> rowBlk, colBlk, diagInv;  // [9 per block] row-major; L_ii^-1 per node
  // supernodes: the leaves and separators of the dissection, contiguous row
  // ranges in factor order, children before parents; a supernode's rows read
  // only rows of its own range and of its descendants (forward solve)
  std::vector<uint32_t> snStart;  // [supernodes + 1]
  std::vector<int32_t> snChild;   // [2 per supernode] -1: none
  std::vector<int32_t> snParent;  // [supernodes] -1: a root
  // per row: its first block inside its supernode (row view: columns >= the
  // supernode's first row) and its first block past it (column view: rows >=
  // the supernode's end), so that a solve reads the finished supernodes'
  // values in one pass and its own rows' one by one
  std::vector<uint32_t> rowSplit, colSplit;

  uint64_t factorNonZeros() const {  // scalar entries of L: 9 per off-diagonal block, 6 per diagonal block
    return ready ? uint64_t(9) * rowCol.size() + uint64_t(6) * nodes : 0u;
  }

  // Order and symbolic factor of a mesh: tets [4 T] node ids, rest [3 V].
  void analyze(uint32_t V, const uint8_t* anchored, const std::vector<uint32_t>& tets, const double* rest) {
    nodes = V;
    const size_t T = tets.size() / 4;
    // free-free couplings, both directions, without the node itself
    std::vector<std::vector<uint32_t>> adj(V);
    for (size_t e = 0; e < T; ++e)
      for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b) {
          const uint32_t na = tets[4 * e + a], nb = tets[4 * e + b];
          if (na != nb && !anchored[na] && !anchored[nb]) adj[na].push_back(nb);
        }
    uint64_t stored = 0;
    for (uint32_t v = 0; v < V; ++v) {
      auto& l = adj[v];
      std::sort(l.begin(), l.end());
      l.erase(std::unique(l.begin(), l.end()), l.end());
      stored += 9u * l.size() + (anchored[v] ? 3u : 9u);
    }
    // a free node outside every tet holds its 3 diagonal entries only
    std::vector<uint8_t> inTet(V, 0);
    for (size_t e = 0; e < T; ++e)
      for (int a = 0; a < 4; ++a) inTet[tets[4 * e + a]] = 1;
    for (uint32_t v = 0; v < V; ++v)
      if (!anchored[v] && !inTet[v]) stored -= 6u;
    systemNonZeros = stored;
    // ---- order: anchored nodes first (they couple to nothing), then nested dissection
    perm.clear();
    perm.reserve(V);
    snStart.assign(1, 0u);
    snChild.clear();
    std::vector<uint32_t> free;
    for (uint32_t v = 0; v < V; ++v) (anchored[v] ? perm : free).push_back(v);
    if (!perm.empty()) addSupernode(-1, -1);  // the anchored rows: no entries
    std::vector<uint32_t> mark(V, 0u);
    uint32_t stamp = 0;
    dissect(free, adj, rest, mark, stamp);
    snParent.assign(snStart.size() - 1, -1);
    for (size_t p = 0; p + 1 < snStart.size(); ++p)
      for (int c = 0; c < 2; ++c)
        if (snChild[2 * p + c] >= 0) snParent[snChild[2 * p + c]] = int32_t(p);
    iperm.assign(V, 0u);
    for (uint32_t i = 0; i < V; ++i) iperm[perm[i]] = i;
    // ---- elimination tree (Liu, with path compression) and row patterns
    std::vector<std::vector<uint32_t>> lower(V);  // neighbours of i earlier in the order
    for (uint32_t v = 0; v < V; ++v)
      for (uint32_t w : adj[v])
        if (iperm[w] < iperm[v]) lower[iperm[v]].push_back(iperm[w]);
    const uint32_t NONE = ~0u;
    std::vector<uint32_t> parent(V, NONE), ancestor(V, NONE);
    for (uint32_t i = 0; i < V; ++i)
      for (uint32_t k : lower[i]) {
        uint32_t r = k;
        while (ancestor[r] != NONE && ancestor[r] != i) {
          const uint32_t next = ancestor[r];
          ancestor[r] = i;
          r = next;
        }
        if (ancestor[r] == NONE) {
          ancestor[r] = i;
          parent[r] = i;
        }
      }
    rowStart.assign(V + 1, 0u);
    rowCol.clear();
    std::vector<uint32_t> seen(V, NONE), pattern;
    for (uint32_t i = 0; i < V; ++i) {
      pattern.clear();
      seen[i] = i;
      for (uint32_t k : lower[i])
        for (uint32_t r = k; seen[r] != i; r = parent[r]) {  // the path up to a node already reached
          seen[r] = i;
          pattern.push_back(r);
        }
      std::sort(pattern.begin(), pattern.end());
      rowCol.insert(rowCol.end(), pattern.begin(), pattern.end());
      rowStart[i + 1] = uint32_t(rowCol.size());
    }
    // ---- the column view
    colStart.assign(V + 1, 0u);
    for (uint32_t c : rowCol) ++colStart[c + 1];
    for (uint32_t i = 0; i < V; ++i) colStart[i + 1] += colStart[i];
    colRow.assign(rowCol.size(), 0u);
    std::vector<uint32_t> fill(colStart.begin(), colStart.end() - 1);
    for (uint32_t i = 0; i < V; ++i)
      for (uint32_t k = rowStart[i]; k < rowStart[i + 1]; ++k) colRow[fill[rowCol[k]]++] = i;
    rowSplit.assign(V, 0u);
    colSplit.assign(V, 0u);
    for (size_t p = 0; p + 1 < snStart.size(); ++p)
      for (uint32_t i = snStart[p]; i < snStart[p + 1]; ++i) {
        rowSplit[i] = uint32_t(std::lower_bound(rowCol.begin() + rowStart[i], rowCol.begin() + rowStart[i + 1],
                                                snStart[p]) - rowCol.begin());
        colSplit[i] = uint32_t(std::lower_bound(colRow.begin() + colStart[i], colRow.begin() + colStart[i + 1],
                                                snStart[p + 1]) - colRow.begin());
      }
    analyzed = true;
  }

  // A supernode of the rows appended to perm since the last one.
  int32_t addSupernode(int32_t a, int32_t b) {
    snStart.push_back(uint32_t(perm.size()));
    snChild.push_back(a);
    snChild.push_back(b);
    return int32_t(snStart.size()) - 2;
  }
  // Nested dissection of a free node set: split at the median of the widest
  // coordinate, the separator being the lower side's nodes that touch the
  // upper side; the two sides first, the separator last.  Returns the
  // subtree's supernode (-1 for an empty set).
  int32_t dissect(std::vector<uint32_t>& set, const std::vector<std::vector<uint32_t>>& adj, const double* rest,
                  std::vector<uint32_t>& mark, uint32_t& stamp) {
    constexpr size_t LEAF = 64;
    if (set.empty()) return -1;
    if (set.size() <= LEAF) {
      perm.insert(perm.end(), set.begin(), set.end());
      return addSupernode(-1, -1);
    }
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (uint32_t v : set)
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(lo[k], rest[3 * size_t(v) + k]);
        hi[k] = std::max(hi[k], rest[3 * size_t(v) + k]);
      }
    int axis = 0;
    for (int k = 1; k < 3; ++k)
      if (hi[k] - lo[k] > hi[axis] - lo[axis]) axis = k;
    const size_t half = set.size() / 2;
    std::nth_element(set.begin(), set.begin() + half, set.end(), [&](uint32_t a, uint32_t b) {
      const double ca = rest[3 * size_t(a) + axis], cb = rest[3 * size_t(b) + axis];
      return ca < cb || (ca == cb && a < b);
    });
    const uint32_t upper = ++stamp;
    for (size_t k = half; k < set.size(); ++k) mark[set[k]] = upper;
    std::vector<uint32_t> left, right(set.begin() + half, set.end()), sep;
    for (size_t k = 0; k < half; ++k) {
      const uint32_t v = set[k];
      bool touches = false;
      for (uint32_t w : adj[v])
        if (mark[w] == upper) {
          touches = true;
          break;
        }
      (touches ? sep : left).push_back(v);
    }
    std::vector<uint32_t>().swap(set);
    const int32_t a = dissect(left, adj, rest, mark, stamp);
    const int32_t b = dissect(right, adj, rest, mark, stamp);
    perm.insert(perm.end(), sep.begin(), sep.end());
    return addSupernode(a, b);
  }

  // Numeric factor.  diag [9 V] and the element blocks blocks[16 per tet][9]
  // (row-major, block (a, b) of tet e at 16 e + 4 a + b) in node numbering;
  // couplings that touch an anchored node are left out.  False when a pivot
  // block is not positive definite (SimplicialLLT's NumericalIssue).
  bool factor(const uint8_t* anchored, const std::vector<uint32_t>& tets, const std::vector<double>& blocks,
              const std::vector<double>& diag) {
    const uint32_t V = nodes;
    const size_t T = tets.size() / 4;
    rowBlk.assign(size_t(9) * rowCol.size(), 0.0);
    colBlk.assign(size_t(9) * rowCol.size(), 0.0);
    diagInv.assign(size_t(9) * V, 0.0);
    std::vector<double> permDia(size_t(9) * V);
    for (uint32_t v = 0; v < V; ++v) std::copy_n(&diag[9 * size_t(v)], 9, &permDia[9 * size_t(iperm[v])]);
    // the lower blocks of P A P^T into their places in the row pattern
    for (size_t e = 0; e < T; ++e)
      for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b) {
          const uint32_t na = tets[4 * e + a], nb = tets[4 * e + b];
          if (anchored[na] || anchored[nb]) continue;
          const uint32_t i = iperm[na], j = iperm[nb];
          const double* B = &blocks[9 * (16 * e + 4 * a + b)];
          if (i == j) {
            for (int q = 0; q < 9; ++q) permDia[9 * size_t(i) + q] += B[q];
          } else if (j < i) {
            const uint32_t* c0 = &rowCol[rowStart[i]];
            const uint32_t k = rowStart[i] + uint32_t(std::lower_bound(c0, c0 + (rowStart[i + 1] - rowStart[i]), j) - c0);
            for (int q = 0; q < 9; ++q) rowBlk[9 * size_t(k) + q] += B[q];
          }
        }
    std::vector<uint32_t> colFill(colStart.begin(), colStart.end() - 1);
    // One row of the up-looking factor; `where` is the caller's scratch.  Rows
    // of supernodes in disjoint subtrees touch disjoint columns, so the
    // supernodes of one depth of the dissection are factored in parallel.
    const auto factorRow = [&](uint32_t i, std::vector<uint32_t>& where) -> bool {
      const uint32_t k0 = rowStart[i], k1 = rowStart[i + 1];
      for (uint32_t k = k0; k < k1; ++k) where[rowCol[k]] = k;
      double d[9];
      std::copy_n(&permDia[9 * size_t(i)], 9, d);
      for (uint32_t k = k0; k < k1; ++k) {
        const uint32_t j = rowCol[k];
        double* x = &rowBlk[9 * size_t(k)];
        // L_ij = x_j L_jj^-T
        const double* Di = &diagInv[9 * size_t(j)];
        double l[9];
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) l[3 * r + c] = x[3 * r] * Di[3 * c] + x[3 * r + 1] * Di[3 * c + 1] + x[3 * r + 2] * Di[3 * c + 2];
        std::copy_n(l, 9, x);
        // x_m -= L_ij L_mj^T for the rows m of column j before i
        for (uint32_t p = colStart[j]; p < colFill[j]; ++p) {
          double* xm = &rowBlk[9 * size_t(where[colRow[p]])];
          const double* lm = &colBlk[9 * size_t(p)];
          for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
              xm[3 * r + c] -= l[3 * r] * lm[3 * c] + l[3 * r + 1] * lm[3 * c + 1] + l[3 * r + 2] * lm[3 * c + 2];
        }
        // D -= L_ij L_ij^T
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) d[3 * r + c] -= l[3 * r] * l[3 * c] + l[3 * r + 1] * l[3 * c + 1] + l[3 * r + 2] * l[3 * c + 2];
      }
      // L_ii = chol(D), lower; its inverse
      double L[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      if (!(d[0] > 0.0)) return false;
      L[0] = std::sqrt(d[0]);
      L[3] = d[3] / L[0];
      L[6] = d[6] / L[0];
      const double d4 = d[4] - L[3] * L[3];
      if (!(d4 > 0.0)) return false;
      L[4] = std::sqrt(d4);
      L[7] = (d[7] - L[6] * L[3]) / L[4];
      const double d8 = d[8] - L[6] * L[6] - L[7] * L[7];
      if (!(d8 > 0.0)) return false;
      L[8] = std::sqrt(d8);
      double* I = &diagInv[9 * size_t(i)];
      I[0] = 1.0 / L[0];
      I[4] = 1.0 / L[4];
      I[8] = 1.0 / L[8];
      I[3] = -L[3] * I[0] / L[4];
      I[7] = -L[7] * I[4] / L[8];
      I[6] = -(L[6] * I[0] + L[7] * I[3]) / L[8];
      // row i's blocks join their columns
      for (uint32_t k = k0; k < k1; ++k) {
        const uint32_t p = colFill[rowCol[k]]++;
        std::copy_n(&rowBlk[9 * size_t(k)], 9, &colBlk[9 * size_t(p)]);
      }
      return true;
    };
    const size_t S = snParent.size();
    std::vector<uint32_t> depth(S, 0u);
    uint32_t deepest = 0;
    for (size_t p = S; p-- > 0;) {  // parents come after their children
      depth[p] = snParent[p] >= 0 ? depth[snParent[p]] + 1u : 0u;
      deepest = std::max(deepest, depth[p]);
    }
    std::vector<std::vector<uint32_t>> level(size_t(deepest) + 1);
    for (size_t p = 0; p < S; ++p) level[depth[p]].push_back(uint32_t(p));
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    std::atomic<bool> failed{false};
    for (size_t d = level.size(); d-- > 0;) {
      const std::vector<uint32_t>& here = level[d];
      std::atomic<size_t> next{0};
      const auto work = [&]() {
        std::vector<uint32_t> where(V, 0u);
        for (size_t q; (q = next.fetch_add(1)) < here.size();)
          for (uint32_t i = snStart[here[q]]; i < snStart[here[q] + 1]; ++i)
            if (!factorRow(i, where)) {
              failed = true;
              return;
            }
      };
      const unsigned n = unsigned(std::min<size_t>(hw, here.size()));
      if (n <= 1) {
        work();
      } else {
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < n; ++t) pool.emplace_back(work);
        for (std::thread& t : pool) t.join();
      }
      if (failed) return ready = false;
    }
    return ready = true;
  }
};

}  // namespace tl
