"""State transfer across the C ABI (tl_state_set / tl_state_get, the
reference's DeformableState, mesh.h:56-62): element state in the caller's
per-tet layout, converted to the element planes on the device.

* A state read back after a few plastic steps and written into a fresh
  system reads back unchanged: exactly in FP64, within FP32 rounding through
  f32 host buffers.
* A non-symmetric plastic strain is stored as its symmetric part (the
  off-diagonals averaged), as the element planes hold a symmetric tensor.
"""
import numpy as np
import pytest

import talus_b200 as tb
from talus_b200 import _capi as capi
from tests.helpers import DT, GRAVITY, plastic_block

pytestmark = pytest.mark.gpu

FIELDS = ("position", "velocity", "acceleration", "rotation", "plastic")


def stepped_state(precision):
    mesh, mat = plastic_block()
    s = tb.System(mesh, [mat], precision)
    s.set_state(tb.rest_state(mesh))
    for _ in range(4):
        s.step(tb.Settings(), GRAVITY, DT)
    st = s.get_state()
    s.close()
    assert np.abs(st.plastic).max() > 0.0  # the block has yielded
    return mesh, mat, st


def transfer(system, dtype, arrays):
    dt = np.float64 if dtype == capi.TL_DTYPE_F64 else np.float32
    src = [np.ascontiguousarray(a, dt) for a in arrays]
    capi.check(capi.lib().tl_state_set(system.handle, 0, dtype, *[a.ctypes.data for a in src]), system.context.handle)
    out = [np.zeros_like(a) for a in src]
    capi.check(capi.lib().tl_state_get(system.handle, 0, dtype, *[a.ctypes.data for a in out]), system.context.handle)
    return src, out


@pytest.mark.parametrize("precision", [tb.FP64, tb.FP32_MIXED])
@pytest.mark.parametrize("dtype", [capi.TL_DTYPE_F64, capi.TL_DTYPE_F32])
def test_state_round_trip(precision, dtype):
    mesh, mat, st = stepped_state(precision)
    s = tb.System(mesh, [mat], precision)
    src, out = transfer(s, dtype, [getattr(st, f) for f in FIELDS])
    s.close()
    exact = precision == tb.FP64 and dtype == capi.TL_DTYPE_F64
    for name, a, b in zip(FIELDS, src, out):
        if name in ("rotation", "plastic"):
            tol = 0.0 if exact else 1e-7 * max(np.abs(a).max(), 1e-30)
            assert np.abs(a - b).max() <= tol, name
        if name == "position":
            scale = np.abs(a).max()
            assert np.abs(a - b).max() <= (1e-15 if exact else 2e-7) * scale, name


def test_plastic_strain_is_stored_symmetric():
    mesh, mat, st = stepped_state(tb.FP64)
    rng = np.random.default_rng(5)
    plastic = st.plastic.copy()
    plastic[:, :9] += 1e-4 * rng.standard_normal((mesh.tets, 9))
    s = tb.System(mesh, [mat], tb.FP64)
    arrays = [getattr(st, f) for f in FIELDS[:4]] + [plastic]
    _, out = transfer(s, capi.TL_DTYPE_F64, arrays)
    s.close()
    e = plastic[:, :9].reshape(-1, 3, 3)
    sym = 0.5 * (e + np.transpose(e, (0, 2, 1)))
    got = out[4][:, :9].reshape(-1, 3, 3)
    assert np.abs(got - sym).max() <= 1e-15 * np.abs(sym).max()
    assert np.array_equal(out[4][:, 9], plastic[:, 9])
