"""Host builder of the assembled operator's sliced-ELL structure
(talus_b200/csrc/tl_sell_build.h), compiled with g++ and checked on the CPU.

A small driver restates on the host what the device does with the structure:
the diagonal blocks written by kNodeAssemble (each node's corner blocks
summed), the symmetric assembly of kSellAssemble (each block above the
diagonal summed from its contributors, its transpose written at the mirror
position) and the row matvec of kPcgSell, for random symmetric 12x12 element
matrices.
The result must equal the element-by-element product
y = sum_e K_e p_e (solver.cc:904-1048 applies the operator that way), on a
Kuhn box and on a box with elements removed (uneven rows and slices).
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import talus_b200 as tb

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "talus_b200", "csrc")

DRIVER = r"""
#include "tl_sell_build.h"
#include <cmath>
#include <cstdio>
#include <vector>
using namespace tl;
int main(int argc, char** argv) {
  FILE* f = std::fopen(argv[1], "rb");
  uint32_t rows, T, E;
  if (std::fread(&rows, 4, 1, f) != 1 || std::fread(&T, 4, 1, f) != 1 || std::fread(&E, 4, 1, f) != 1) return 2;
  std::vector<uint32_t> tets(4 * size_t(T)), start(size_t(rows) + 1), entry(E);
  if (std::fread(tets.data(), 4, tets.size(), f) != tets.size()) return 2;
  if (std::fread(start.data(), 4, start.size(), f) != start.size()) return 2;
  if (std::fread(entry.data(), 4, entry.size(), f) != entry.size()) return 2;
  std::vector<double> K(size_t(T) * 144), p(3 * size_t(rows));
  if (std::fread(K.data(), 8, K.size(), f) != K.size()) return 2;
  if (std::fread(p.data(), 8, p.size(), f) != p.size()) return 2;
  std::fclose(f);
  SellHost h = buildSellHost(rows, tets.data(), start, entry);
  // diagonal blocks as kNodeAssemble writes them: each node's corner blocks
  std::vector<double> val(size_t(h.positions) * 9, 0.0);
  for (uint32_t e = 0; e < T; ++e)
    for (int a = 0; a < 4; ++a) {
      const uint32_t pos = h.diag[tets[4 * e + a]];
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) val[size_t(pos) * 9 + 3 * r + c] += K[size_t(e) * 144 + (3 * a + r) * 12 + 3 * a + c];
    }
  // the blocks above the diagonal and their transposes, as kSellAssemble writes them
  for (size_t i = 0; i < h.upper.size(); ++i) {
    const uint32_t pos = h.upper[i], mpos = h.mirror[i];
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t q = h.cstart[pos]; q < h.cstart[pos + 1]; ++q) {
      const uint32_t code = h.centry[q], e = code >> 4, a = (code >> 2) & 3u, b = code & 3u;
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) acc[3 * r + c] += K[size_t(e) * 144 + (3 * a + r) * 12 + 3 * b + c];
    }
    for (int c = 0; c < 9; ++c) val[size_t(pos) * 9 + c] = acc[c];
    if (mpos != pos)
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) val[size_t(mpos) * 9 + 3 * r + c] = acc[3 * c + r];
  }
  // row matvec as kPcgSell does it
  double err = 0, scale = 0;
  std::vector<double> ref(3 * size_t(rows), 0.0);
  for (uint32_t e = 0; e < T; ++e)
    for (int a = 0; a < 4; ++a)
      for (int r = 0; r < 3; ++r) {
        double s = 0;
        for (int b = 0; b < 4; ++b)
          for (int c = 0; c < 3; ++c) s += K[size_t(e) * 144 + (3 * a + r) * 12 + 3 * b + c] * p[3 * tets[4 * e + b] + c];
        ref[3 * tets[4 * e + a] + r] += s;
      }
  for (uint32_t row = 0; row < rows; ++row) {
    const uint32_t sl = row / SELL_ROWS, lane = row % SELL_ROWS;
    double y[3] = {0, 0, 0};
    for (uint32_t pos = h.sliceStart[sl] + lane; pos < h.sliceStart[sl + 1]; pos += SELL_ROWS) {
      if (h.groupSlice[pos / SELL_ROWS] != sl) return 3;
      const uint32_t c = h.col[pos];
      for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) y[r] += val[size_t(pos) * 9 + 3 * r + k] * p[3 * size_t(c) + k];
    }
    for (int r = 0; r < 3; ++r) {
      err = std::fmax(err, std::fabs(y[r] - ref[3 * size_t(row) + r]));
      scale = std::fmax(scale, std::fabs(ref[3 * size_t(row) + r]));
    }
  }
  for (uint32_t row = 0; row < rows; ++row)
    if (h.col[h.diag[row]] != row) return 4;
  size_t contributors = h.centry.size();
  std::printf("%.17g %.17g %zu %u %u %zu\n", err, scale, contributors, h.positions, h.widest, h.upper.size());
  return 0;
}
"""


def incidence(tets, nodes):
    lists = [[] for _ in range(nodes)]
    for e, t in enumerate(tets):
        for c in range(4):
            lists[int(t[c])].append(4 * e + c)
    start = np.zeros(nodes + 1, np.uint32)
    start[1:] = np.cumsum([len(l) for l in lists])
    return start, np.array([x for l in lists for x in l], np.uint32)


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("sell")
    src = d / "driver.cc"
    src.write_text(DRIVER)
    exe = d / "driver"
    subprocess.run([gxx, "-O1", "-std=c++17", "-I", CSRC, str(src), "-o", str(exe)], check=True)
    return exe, d


def run(driver, tets, nodes, seed):
    exe, d = driver
    tets = np.ascontiguousarray(tets, np.uint32)
    start, entry = incidence(tets, nodes)
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((tets.shape[0], 12, 12))
    K = A + np.transpose(A, (0, 2, 1))  # symmetric element matrices
    p = rng.standard_normal(3 * nodes)
    path = d / f"in{seed}.bin"
    with open(path, "wb") as f:
        np.array([nodes, tets.shape[0], entry.size], np.uint32).tofile(f)
        tets.tofile(f)
        start.tofile(f)
        entry.tofile(f)
        K.astype(np.float64).tofile(f)
        p.astype(np.float64).tofile(f)
    out = subprocess.run([str(exe), str(path)], check=True, capture_output=True, text=True).stdout.split()
    err, scale = float(out[0]), float(out[1])
    return err, scale, int(out[2]), int(out[3]), int(out[4]), int(out[5])


def test_kuhn_box(driver):
    mesh = tb.box_mesh((5, 3, 4), voxel=0.1)
    err, scale, contributors, positions, widest, upper = run(driver, mesh.tet_nodes, mesh.nodes, 1)
    assert err <= 1e-12 * scale
    assert contributors == 16 * mesh.tets  # every (element, corner, corner) once
    assert widest == 15  # an interior Kuhn node has 14 neighbours and itself
    assert positions % 32 == 0


def test_uneven_rows(driver):
    mesh = tb.box_mesh((6, 5, 4), voxel=0.1)
    keep = np.random.default_rng(2).random(mesh.tets) > 0.3  # holes: uneven rows, isolated nodes
    err, scale, contributors, _, _, _ = run(driver, mesh.tet_nodes[keep], mesh.nodes, 3)
    assert err <= 1e-12 * scale
    assert contributors == 16 * int(keep.sum())
