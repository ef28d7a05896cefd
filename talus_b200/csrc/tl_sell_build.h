// Host construction of the sliced-ELL block structure of the PCG operator
// (the device side is tl_sell.cuh).  Plain C++, no CUDA types, so that the
// CPU tests compile it with g++ and check it against an element-by-element
// matvec.
#pragma once

#include <algorithm>
#include <cstdint>
#include <utility>
#include <vector>

namespace tl {

constexpr uint32_t SELL_ROWS = 32;  // rows per slice (one warp)

struct SellHost {
  uint32_t rows = 0, slices = 0, positions = 0, widest = 1;
  std::vector<uint32_t> sliceStart;  // [slices + 1] first block position of each slice
  std::vector<uint32_t> groupSlice;  // [positions / 32] slice of each 32-position group
  std::vector<uint32_t> col;         // [positions] column node (padding: own row, or 0 past the rows)
  std::vector<uint32_t> cstart;      // [positions + 1] contributor range of each position
  std::vector<uint32_t> centry;      // (element << 4) | (row corner << 2) | column corner, ascending element
  std::vector<uint32_t> upper;       // block positions with row < column, longest contributor lists first
  std::vector<uint32_t> mirror;      // position of each upper block's transpose
  std::vector<uint32_t> diag;        // [rows] position of each row's diagonal block
};

// rows: node rows [0, rows); tets4: 4 node ids per element; incStart /
// incEntry: the node -> (4 element + corner) incidence CSR with elements
// ascending per node (the reference's buildIncidence, solver.cc:1065-1101).
// Each row's column slots are its neighbour nodes (the nodes of its
// elements) in ascending order; slices of 32 rows are padded to their
// widest row; block (slot k, lane) of slice s sits at sliceStart[s] + 32 k +
// lane.  A block's contributors are the (element, row corner, column corner)
// triples whose element holds both nodes, in ascending element order.
inline SellHost buildSellHost(uint32_t rows, const uint32_t* tets4, const std::vector<uint32_t>& incStart,
                              const std::vector<uint32_t>& incEntry) {
  SellHost h;
  h.rows = rows;
  const uint32_t slices = (rows + SELL_ROWS - 1) / SELL_ROWS;
  h.slices = slices;
  // neighbours of each row
  std::vector<uint32_t> nbStart(size_t(rows) + 1, 0), nb;
  nb.reserve(size_t(rows) * 16);
  std::vector<uint32_t> tmp;
  for (uint32_t r = 0; r < rows; ++r) {
    tmp.clear();
    for (uint32_t k = incStart[r]; k < incStart[r + 1]; ++k) {
      const uint32_t* t = tets4 + 4 * size_t(incEntry[k] >> 2);
      tmp.insert(tmp.end(), t, t + 4);
    }
    if (tmp.empty()) tmp.push_back(r);
    std::sort(tmp.begin(), tmp.end());
    tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
    nb.insert(nb.end(), tmp.begin(), tmp.end());
    nbStart[r + 1] = uint32_t(nb.size());
  }
  // slices
  h.sliceStart.assign(size_t(slices) + 1, 0);
  for (uint32_t sl = 0; sl < slices; ++sl) {
    uint32_t width = 1;
    for (uint32_t r = sl * SELL_ROWS; r < std::min(rows, (sl + 1) * SELL_ROWS); ++r)
      width = std::max(width, nbStart[r + 1] - nbStart[r]);
    h.sliceStart[sl + 1] = h.sliceStart[sl] + width * SELL_ROWS;
    h.widest = std::max(h.widest, width);
  }
  const uint32_t positions = h.sliceStart[slices];
  h.positions = positions;
  // contributors of (row, slot), ascending element: per row, codes keyed by slot
  std::vector<uint32_t> slotStart(nb.size() + rows + 1, 0), codes;  // per row: slots + 1 offsets
  std::vector<uint32_t> rowSlotBase(size_t(rows) + 1, 0);
  codes.reserve(incEntry.size() * 4);
  std::vector<std::pair<uint32_t, uint32_t>> pairs;
  for (uint32_t r = 0; r < rows; ++r) {
    const uint32_t* nr = nb.data() + nbStart[r];
    const uint32_t len = nbStart[r + 1] - nbStart[r];
    pairs.clear();
    for (uint32_t k = incStart[r]; k < incStart[r + 1]; ++k) {
      const uint32_t e = incEntry[k] >> 2, a = incEntry[k] & 3u;
      const uint32_t* q = tets4 + 4 * size_t(e);
      for (uint32_t b = 0; b < 4; ++b) {
        const uint32_t slot = uint32_t(std::lower_bound(nr, nr + len, q[b]) - nr);
        pairs.emplace_back(slot, (e << 4) | (a << 2) | b);
      }
    }
    std::stable_sort(pairs.begin(), pairs.end(),
                     [](const std::pair<uint32_t, uint32_t>& x, const std::pair<uint32_t, uint32_t>& y) {
                       return x.first < y.first;
                     });
    const uint32_t base = nbStart[r] + r;  // this row's len + 1 offsets
    rowSlotBase[r] = base;
    size_t j = 0;
    for (uint32_t k = 0; k <= len; ++k) {
      slotStart[base + k] = uint32_t(codes.size());
      while (k < len && j < pairs.size() && pairs[j].first == k) codes.push_back(pairs[j++].second);
    }
  }
  // positions in slice order
  h.col.assign(positions, 0);
  h.cstart.assign(size_t(positions) + 1, 0);
  h.groupSlice.assign(positions / SELL_ROWS, 0);
  h.centry.reserve(codes.size());
  for (uint32_t sl = 0; sl < slices; ++sl) {
    const uint32_t width = (h.sliceStart[sl + 1] - h.sliceStart[sl]) / SELL_ROWS;
    for (uint32_t k = 0; k < width; ++k) {
      h.groupSlice[(h.sliceStart[sl] + k * SELL_ROWS) / SELL_ROWS] = sl;
      for (uint32_t lane = 0; lane < SELL_ROWS; ++lane) {
        const uint32_t pos = h.sliceStart[sl] + k * SELL_ROWS + lane, r = sl * SELL_ROWS + lane;
        h.cstart[pos] = uint32_t(h.centry.size());
        if (r >= rows) continue;  // padding row: column 0, zero block
        const uint32_t len = nbStart[r + 1] - nbStart[r];
        if (k >= len) {
          h.col[pos] = r;  // padding slot: own column, zero block
          continue;
        }
        h.col[pos] = nb[nbStart[r] + k];
        const uint32_t* ss = slotStart.data() + rowSlotBase[r];
        h.centry.insert(h.centry.end(), codes.begin() + ss[k], codes.begin() + ss[k + 1]);
      }
    }
  }
  h.cstart[positions] = uint32_t(h.centry.size());
  // blocks above the diagonal and the positions of their transposes; the
  // diagonal positions (their blocks are the node assembly's diagonal blocks)
  h.diag.assign(rows, 0);
  for (uint32_t sl = 0; sl < slices; ++sl) {
    const uint32_t width = (h.sliceStart[sl + 1] - h.sliceStart[sl]) / SELL_ROWS;
    for (uint32_t k = 0; k < width; ++k)
      for (uint32_t lane = 0; lane < SELL_ROWS; ++lane) {
        const uint32_t pos = h.sliceStart[sl] + k * SELL_ROWS + lane, r = sl * SELL_ROWS + lane;
        if (r >= rows || k >= nbStart[r + 1] - nbStart[r]) continue;
        const uint32_t c = h.col[pos];
        if (c == r) h.diag[r] = pos;
        if (c <= r) continue;
        const uint32_t *nc = nb.data() + nbStart[c], *ncEnd = nb.data() + nbStart[c + 1];
        const uint32_t kc = uint32_t(std::lower_bound(nc, ncEnd, r) - nc);
        h.upper.push_back(pos);
        h.mirror.push_back(h.sliceStart[c / SELL_ROWS] + kc * SELL_ROWS + c % SELL_ROWS);
      }
  }
  {  // longest contributor lists first, so warps take similar loop counts
    std::vector<uint32_t> order(h.upper.size());
    for (uint32_t i = 0; i < order.size(); ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
      return h.cstart[h.upper[x] + 1] - h.cstart[h.upper[x]] > h.cstart[h.upper[y] + 1] - h.cstart[h.upper[y]];
    });
    std::vector<uint32_t> u2(h.upper.size()), m2(h.upper.size());
    for (uint32_t i = 0; i < order.size(); ++i) {
      u2[i] = h.upper[order[i]];
      m2[i] = h.mirror[order[i]];
    }
    h.upper.swap(u2);
    h.mirror.swap(m2);
  }
  return h;
}

}  // namespace tl
