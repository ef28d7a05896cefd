"""The host side of the solver state's factor (talus_b200/csrc/tl_factor_host.h),
compiled with g++ and checked on the CPU: the block Cholesky solves its
system, and the damping blocks are the oracle's damping operator
(applyDamping, factor.cc:843-853) applied to the unit directions."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import pyoracle as po
from tests.test_device_math_host import CSRC, CUDA_INCLUDE

SOURCE = r"""
#include "tl_factor_host.h"
using namespace tl;
extern "C" {
void fh_damping_blocks(const double* x, const double* R, const double* Dm, double volume, double youngs,
                       double poisson, double* out) {
  factorDampingBlocks(x, R, Dm, volume, youngs, poisson, out);
}
// A lattice of nx*ny*nz nodes, 6 tets per cube, the j == 0 plane anchored, random SPD element blocks:
// the factor's solve of A x = b against A x, max |A x - b| / max |b|.
// The supernode order the device solves rely on: the supernodes cover the rows
// once in order, every parent comes after its children, and every block of a
// row's L lies in the row's own supernode or a descendant of it.  0 if it
// holds; otherwise the number of violations.
int fh_supernode_violations(int nx, int ny, int nz);
double fh_solve_residual(int nx, int ny, int nz, unsigned seed) {
  const uint32_t V = nx * ny * nz;
  std::vector<double> rest(3 * V);
  std::vector<uint8_t> anch(V, 0);
  auto id = [&](int i, int j, int k) { return uint32_t(i + nx * (j + ny * k)); };
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const uint32_t v = id(i, j, k);
        rest[3 * v] = i; rest[3 * v + 1] = j; rest[3 * v + 2] = k;
        anch[v] = j == 0;
      }
  std::vector<uint32_t> tets;
  const int T6[6][4] = {{0, 1, 3, 7}, {0, 1, 5, 7}, {0, 2, 3, 7}, {0, 2, 6, 7}, {0, 4, 5, 7}, {0, 4, 6, 7}};
  for (int k = 0; k + 1 < nz; ++k)
    for (int j = 0; j + 1 < ny; ++j)
      for (int i = 0; i + 1 < nx; ++i) {
        uint32_t c[8];
        for (int q = 0; q < 8; ++q) c[q] = id(i + (q & 1), j + ((q >> 1) & 1), k + ((q >> 2) & 1));
        for (auto& t : T6) for (int q = 0; q < 4; ++q) tets.push_back(c[t[q]]);
      }
  const size_t T = tets.size() / 4;
  uint64_t st = seed * 2654435761u + 1;
  auto rnd = [&]() { st = st * 6364136223846793005ull + 1442695040888963407ull; return double(st >> 11) / 9007199254740992.0 - 0.5; };
  std::vector<double> blocks(144 * T), diag(9 * V, 0.0);
  for (size_t e = 0; e < T; ++e) {
    double B[12][12];
    for (auto& r : B) for (auto& x : r) x = rnd();
    for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) {
      double s = 0; for (int q = 0; q < 12; ++q) s += B[3 * a + r][q] * B[3 * b + c][q];
      blocks[9 * (16 * e + 4 * a + b) + 3 * r + c] = s;
    }
  }
  for (uint32_t v = 0; v < V; ++v) for (int q = 0; q < 3; ++q) diag[9 * v + 4 * q] = anch[v] ? 1.0 : 2.0;
  BlockFactor f;
  f.analyze(V, anch.data(), tets, rest.data());
  if (!f.factor(anch.data(), tets, blocks, diag)) return -1.0;
  std::vector<double> b(3 * V), y(3 * V), w(3 * V), x(3 * V), ax(3 * V, 0.0);
  for (auto& q : b) q = rnd();
  for (uint32_t i = 0; i < V; ++i) {  // forward, factor order
    double acc[3] = {0, 0, 0};
    for (uint32_t k = f.rowStart[i]; k < f.rowStart[i + 1]; ++k) {
      const double* L = &f.rowBlk[9 * k]; const double* yj = &y[3 * f.rowCol[k]];
      for (int r = 0; r < 3; ++r) acc[r] += L[3 * r] * yj[0] + L[3 * r + 1] * yj[1] + L[3 * r + 2] * yj[2];
    }
    const double* D = &f.diagInv[9 * i]; const double* bo = &b[3 * f.perm[i]];
    const double bb[3] = {bo[0] - acc[0], bo[1] - acc[1], bo[2] - acc[2]};
    y[3 * i] = D[0] * bb[0]; y[3 * i + 1] = D[3] * bb[0] + D[4] * bb[1]; y[3 * i + 2] = D[6] * bb[0] + D[7] * bb[1] + D[8] * bb[2];
  }
  for (uint32_t i = V; i-- > 0;) {  // backward
    double acc[3] = {0, 0, 0};
    for (uint32_t k = f.colStart[i]; k < f.colStart[i + 1]; ++k) {
      const double* L = &f.colBlk[9 * k]; const double* wj = &w[3 * f.colRow[k]];
      for (int a = 0; a < 3; ++a) acc[a] += L[a] * wj[0] + L[3 + a] * wj[1] + L[6 + a] * wj[2];
    }
    const double* D = &f.diagInv[9 * i];
    const double bb[3] = {y[3 * i] - acc[0], y[3 * i + 1] - acc[1], y[3 * i + 2] - acc[2]};
    w[3 * i] = D[0] * bb[0] + D[3] * bb[1] + D[6] * bb[2]; w[3 * i + 1] = D[4] * bb[1] + D[7] * bb[2]; w[3 * i + 2] = D[8] * bb[2];
  }
  for (uint32_t v = 0; v < V; ++v) for (int r = 0; r < 3; ++r) x[3 * v + r] = w[3 * f.iperm[v] + r];
  for (uint32_t v = 0; v < V; ++v) for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) ax[3 * v + r] += diag[9 * v + 3 * r + c] * x[3 * v + c];
  for (size_t e = 0; e < T; ++e) for (int a = 0; a < 4; ++a) for (int bq = 0; bq < 4; ++bq) {
    const uint32_t na = tets[4 * e + a], nb = tets[4 * e + bq];
    if (anch[na] || anch[nb]) continue;
    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) ax[3 * na + r] += blocks[9 * (16 * e + 4 * a + bq) + 3 * r + c] * x[3 * nb + c];
  }
  double err = 0, nb = 0;
  for (size_t q = 0; q < 3 * V; ++q) { err = std::max(err, std::abs(ax[q] - b[q])); nb = std::max(nb, std::abs(b[q])); }
  return err / nb;
}
int fh_supernode_violations(int nx, int ny, int nz) {
  const uint32_t V = nx * ny * nz;
  std::vector<double> rest(3 * V);
  std::vector<uint8_t> anch(V, 0);
  auto id = [&](int i, int j, int k) { return uint32_t(i + nx * (j + ny * k)); };
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const uint32_t v = id(i, j, k);
        rest[3 * v] = i; rest[3 * v + 1] = j; rest[3 * v + 2] = k;
        anch[v] = j == 0 || j == ny - 1;
      }
  std::vector<uint32_t> tets;
  const int T6[6][4] = {{0, 1, 3, 7}, {0, 1, 5, 7}, {0, 2, 3, 7}, {0, 2, 6, 7}, {0, 4, 5, 7}, {0, 4, 6, 7}};
  for (int k = 0; k + 1 < nz; ++k)
    for (int j = 0; j + 1 < ny; ++j)
      for (int i = 0; i + 1 < nx; ++i) {
        uint32_t c[8];
        for (int q = 0; q < 8; ++q) c[q] = id(i + (q & 1), j + ((q >> 1) & 1), k + ((q >> 2) & 1));
        for (auto& t : T6) for (int q = 0; q < 4; ++q) tets.push_back(c[t[q]]);
      }
  BlockFactor f;
  f.analyze(V, anch.data(), tets, rest.data());
  const size_t S = f.snParent.size();
  int bad = 0;
  if (f.snStart.front() != 0 || f.snStart.back() != V) ++bad;
  std::vector<int32_t> snOf(V, -1);
  for (size_t p = 0; p < S; ++p) {
    if (f.snStart[p] > f.snStart[p + 1]) ++bad;
    for (uint32_t i = f.snStart[p]; i < f.snStart[p + 1]; ++i) snOf[i] = int32_t(p);
    if (f.snParent[p] >= 0 && f.snParent[p] <= int32_t(p)) ++bad;
    for (int c = 0; c < 2; ++c) {
      const int32_t ch = f.snChild[2 * p + c];
      if (ch >= 0 && f.snParent[ch] != int32_t(p)) ++bad;
    }
  }
  auto within = [&](int32_t a, int32_t p) { for (; a >= 0; a = f.snParent[a]) if (a == p) return true; return false; };
  for (uint32_t i = 0; i < V; ++i)
    for (uint32_t k = f.rowStart[i]; k < f.rowStart[i + 1]; ++k)
      if (!within(snOf[f.rowCol[k]], snOf[i])) ++bad;
  return bad;
}
}
"""


@pytest.fixture(scope="module")
def fh(tmp_path_factory):
    if shutil.which("g++") is None or not os.path.exists(os.path.join(CUDA_INCLUDE, "cuda_runtime.h")):
        pytest.skip("g++ or the CUDA headers are missing")
    d = tmp_path_factory.mktemp("factor_host")
    src, lib = d / "fh.cc", d / "libfh.so"
    src.write_text(SOURCE)
    subprocess.run(["g++", "-std=c++17", "-O2", "-shared", "-fPIC", "-Wno-unknown-pragmas", f"-I{CUDA_INCLUDE}",
                    f"-I{CSRC}", "-o", str(lib), str(src)], check=True)
    handle = C.CDLL(str(lib))
    handle.fh_damping_blocks.argtypes = [C.c_void_p] * 3 + [C.c_double] * 3 + [C.c_void_p]
    handle.fh_solve_residual.argtypes = [C.c_int, C.c_int, C.c_int, C.c_uint]
    handle.fh_solve_residual.restype = C.c_double
    handle.fh_supernode_violations.argtypes = [C.c_int, C.c_int, C.c_int]
    return handle


@pytest.mark.parametrize("dims", [(3, 3, 3), (6, 5, 5), (12, 6, 6)])
def test_block_factor_solves_its_system(fh, dims):
    assert fh.fh_solve_residual(*dims, 7) <= 1e-10


@pytest.mark.parametrize("dims", [(3, 3, 3), (17, 9, 9), (9, 17, 5), (33, 17, 17)])
def test_supernodes_order_the_solves(fh, dims):
    """The device solves hand supernodes out children first (forward) and
    parents first (backward), each waiting on the supernodes it reads: that
    needs every row's blocks to lie in its own supernode or below it."""
    assert fh.fh_supernode_violations(*dims) == 0


def test_damping_blocks_are_the_oracle_damping_operator(fh):
    rng = np.random.default_rng(3)
    for _ in range(5):
        rest = np.array([[0, 0, 0], [0.1, 0, 0], [0, 0.1, 0], [0, 0, 0.1]]) + rng.uniform(-0.01, 0.01, (4, 3))
        dm = np.linalg.inv((rest[1:] - rest[0]).T)
        volume = abs(np.linalg.det((rest[1:] - rest[0]).T)) / 6.0
        corners = rest + rng.uniform(-0.02, 0.02, (4, 3))
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        rot = q * np.sign(np.linalg.det(q))
        mat = po.material(1000.0, 2e6, 0.35, 0.02)
        got = np.zeros(144)
        a = [np.ascontiguousarray(x, np.float64) for x in (corners, rot, dm)]
        fh.fh_damping_blocks(a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, volume, 2e6, 0.35,
                             got.ctypes.data)
        blocks = got.reshape(4, 4, 3, 3)
        for corner in range(4):
            for axis in range(3):
                unit = np.zeros((4, 3))
                unit[corner, axis] = 1.0
                want = po.damping_apply(po.F64, corners, rot, dm, volume, mat, unit)
                col = blocks[:, corner, :, axis]
                assert np.abs(col - want).max() <= 1e-10 * max(1.0, np.abs(want).max())
