"""The kernels' 3x3 math (talus_b200/csrc/tl_math.cuh) compiled for the host
with g++ and checked against the oracle on the CPU.

tl_math.cuh is host-device code: the element rotations (polar iteration,
material.cc:168-197; the invertible rotation of an inverted tet,
material.cc:24-64), volumeChange (J - 1 without cancellation) and the
finite-strain return map (plasticflow.cc:110-150) that the element pass and
the flow kernel call.  Built here into a small shared library, the same
source runs on seeded matrices beside the oracle's restatements.  The
arithmetic differs only by FMA contraction, so the bars are 1e-12 (one-shot
formulas) and 1e-9 (the iterations, whose stop tests may fall one pass
apart).
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import pyoracle as po

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "talus_b200", "csrc")
CUDA_INCLUDE = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")

SOURCE = r"""
#include "tl_math.cuh"
using namespace tl;
static M3<double> load(const double* a) {
  M3<double> m;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) m.m[i][j] = a[3 * i + j];
  return m;
}
static void store(const M3<double>& m, double* a) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a[3 * i + j] = m.m[i][j];
}
extern "C" {
void dm_rotation(const double* f, int invertible, double* out) { store(elementRotation(load(f), invertible != 0), out); }
double dm_volume_change(const double* h) { return volumeChange(load(h)); }
int dm_hencky_return(const double* fe, double shear, double yield, double* out, double* strain, double* trial) {
  M3<double> back;
  double s = 0.0, t = 0.0;
  if (!henckyReturn(load(fe), shear, yield, back, s, t)) return 0;
  store(back, out);
  *strain = s;
  *trial = t;
  return 1;
}
}
"""


@pytest.fixture(scope="module")
def dm(tmp_path_factory):
    if shutil.which("g++") is None or not os.path.exists(os.path.join(CUDA_INCLUDE, "cuda_runtime.h")):
        pytest.skip("g++ or the CUDA headers are missing")
    d = tmp_path_factory.mktemp("device_math")
    src, lib = d / "dm.cc", d / "libdm.so"
    src.write_text(SOURCE)
    subprocess.run(["g++", "-std=c++17", "-O2", "-shared", "-fPIC", "-Wno-unknown-pragmas", f"-I{CUDA_INCLUDE}",
                    f"-I{CSRC}", "-o", str(lib), str(src)], check=True)
    handle = C.CDLL(str(lib))
    handle.dm_rotation.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    handle.dm_volume_change.argtypes = [C.c_void_p]
    handle.dm_volume_change.restype = C.c_double
    handle.dm_hencky_return.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
    return handle


def ptr(a):
    return a.ctypes.data


def gradients(count=200, seed=17):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        f = np.eye(3) + (0.02, 0.2, 0.6)[k % 3] * rng.standard_normal((3, 3))
        if k % 5 == 0:
            f = f @ np.diag([1.0, 1.0, -0.4])  # inverted
        out.append(np.ascontiguousarray(f))
    return out


def test_rotations_match_the_oracle(dm):
    worst = 0.0
    for f in gradients():
        for invertible in (0, 1):
            got = np.zeros((3, 3))
            dm.dm_rotation(ptr(f), invertible, ptr(got))
            mode = po.ROTATION_INVERTIBLE if invertible else po.ROTATION_POLAR
            worst = max(worst, float(np.abs(got - po.rotation(po.F64, f, mode)).max()))
            if invertible:
                assert np.linalg.det(got) > 0.999  # a proper rotation, inverted tets included
    assert worst <= 1e-9, worst


def det_minus_one_exact(h):
    """det(I + H) - 1 in exact rational arithmetic on the FP64 entries of H."""
    from fractions import Fraction

    f = [[Fraction(float(h[i, j])) + (1 if i == j else 0) for j in range(3)] for i in range(3)]
    det = (f[0][0] * (f[1][1] * f[2][2] - f[1][2] * f[2][1]) - f[0][1] * (f[1][0] * f[2][2] - f[1][2] * f[2][0])
           + f[0][2] * (f[1][0] * f[2][1] - f[1][1] * f[2][0]))
    return float(det - 1)


def test_volume_change_is_det_minus_one_without_cancellation(dm):
    rng = np.random.default_rng(3)
    for scale in (1e-9, 1e-6, 1e-3, 0.1, 0.5):
        h = np.ascontiguousarray(scale * rng.standard_normal((3, 3)))
        exact = det_minus_one_exact(h)
        got = dm.dm_volume_change(ptr(h))
        # relative accuracy holds for tiny H, where det(I + H) - 1 in FP64 keeps only a few digits
        assert abs(got - exact) <= 1e-14 * abs(exact), (scale, got, exact)
        naive = np.linalg.det(np.eye(3) + h) - 1.0
        if scale <= 1e-6:
            assert abs(naive - exact) > abs(got - exact)


def test_finite_strain_return_matches_the_oracle(dm):
    rng = np.random.default_rng(9)
    mapped = 0
    for k in range(200):
        fe = np.ascontiguousarray(np.eye(3) + (0.001, 0.01, 0.1)[k % 3] * rng.standard_normal((3, 3)))
        if np.linalg.det(fe) <= 0:
            continue
        shear, yield_stress = 1.0e5, 2.0e3
        out, strain, trial = np.zeros((3, 3)), np.zeros(1), np.zeros(1)
        ok = dm.dm_hencky_return(ptr(fe), shear, yield_stress, ptr(out), ptr(strain), ptr(trial))
        ref = po.hencky_return(fe, shear, yield_stress)
        assert bool(ok) == (ref is not None), k
        if ok:
            mapped += 1
            back, rstrain, rtrial = ref
            assert np.abs(out - back).max() <= 1e-12, k
            assert abs(strain[0] - rstrain) <= 1e-12 * max(1.0, abs(rstrain))
            assert abs(trial[0] - rtrial) <= 1e-9 * rtrial
    assert mapped > 50
