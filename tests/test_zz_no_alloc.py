"""tl_step_noalloc: the step for callers that cannot allocate device memory.

Some callers may not call cudaMalloc at all: an engine frame loop with a fixed
GPU budget, code that runs while a CUDA graph is being captured, a host that
hands out device memory only through its own pool.  tl_step_noalloc keeps all
of its scratch in one fixed array inside the library.  These tests check that
two calls in a row give the same state as the ordinary entry point
(tl_step_host on a resident FP64 system), and that inputs beyond the fixed
capacity are refused.  The file runs last so that a failure here never hides
the rest of the suite, and it passes alone in a fresh process too.
"""
import ctypes as C

import numpy as np
import pytest

import talus_b200 as tb
from talus_b200 import _capi as capi
from talus_b200.deformable import _Body
from tests.helpers import DT, GRAVITY, elastic_block, relative_error


def host_arrays(mesh):
    s = tb.rest_state(mesh)
    return {k: np.ascontiguousarray(getattr(s, k), np.float64) for k in
            ("position", "velocity", "acceleration", "rotation", "plastic")}


def call_noalloc(body, arrays, settings, report):
    g = np.asarray(GRAVITY, np.float64)
    return capi.lib().tl_step_noalloc(0, C.byref(body.desc), capi.TL_DTYPE_F64, arrays["position"].ctypes.data,
                                      arrays["velocity"].ctypes.data, arrays["acceleration"].ctypes.data,
                                      arrays["rotation"].ctypes.data, arrays["plastic"].ctypes.data,
                                      C.byref(settings._c()), g.ctypes.data, DT, C.byref(report))


def call_host(system, arrays, settings, report):
    g = np.asarray(GRAVITY, np.float64)
    return capi.lib().tl_step_host(system.handle, 0, capi.TL_DTYPE_F64, arrays["position"].ctypes.data,
                                   arrays["velocity"].ctypes.data, arrays["acceleration"].ctypes.data,
                                   arrays["rotation"].ctypes.data, arrays["plastic"].ctypes.data,
                                   C.byref(settings._c()), g.ctypes.data, DT, C.byref(report))


@pytest.mark.gpu
@pytest.mark.parametrize("law", [tb.COROTATED, tb.NEO_HOOKEAN])
def test_noalloc_step_matches_the_resident_step_on_two_calls(law):
    mesh, mat = elastic_block()          # 729 nodes, 3072 tets: inside the fixed capacity
    settings = tb.Settings(law=law)
    body = _Body(mesh, [mat])
    mine, ref = host_arrays(mesh), host_arrays(mesh)
    system = tb.System(mesh, [mat], tb.FP64)
    for call in range(2):
        r_mine, r_ref = capi.tl_step_report(), capi.tl_step_report()
        assert call_noalloc(body, mine, settings, r_mine) == capi.TL_OK
        assert call_host(system, ref, settings, r_ref) == capi.TL_OK
        # the FP64 bar of the parity tests: <= 1e-9 relative displacement
        assert relative_error(mine["position"], ref["position"], mesh.rest_positions) <= 1e-9, call
        vscale = np.abs(ref["velocity"]).max()
        assert np.abs(mine["velocity"] - ref["velocity"]).max() <= 1e-9 * vscale, call
        assert np.abs(mine["acceleration"] - ref["acceleration"]).max() <= 1e-9 * np.abs(ref["acceleration"]).max()
        assert r_mine.cg_iterations == r_ref.cg_iterations, call
        assert r_mine.elastic_energy == pytest.approx(r_ref.elastic_energy, rel=1e-9)
    system.close()


@pytest.mark.gpu
def test_noalloc_refuses_the_plastic_newton_loop():
    mesh, _ = elastic_block((4, 4, 4))
    mat = tb.PhysicalMaterial(youngs_modulus=2e7, poissons_ratio=0.35, yield_stress=1e5)
    body = _Body(mesh, [mat])
    arrays = host_arrays(mesh)
    before = arrays["position"].copy()
    rc = call_noalloc(body, arrays, tb.Settings(plastic_passes=40), capi.tl_step_report())
    assert rc == capi.TL_ERR_UNSUPPORTED
    assert np.array_equal(arrays["position"], before)


def test_noalloc_refuses_meshes_beyond_its_capacity():
    """Checked before any device work, so it runs without a GPU too."""
    mesh, mat = elastic_block((11, 11, 11))   # 7986 tets > TL_NOALLOC_MAX_TETS
    assert mesh.tets > 4096
    body = _Body(mesh, [mat])
    arrays = host_arrays(mesh)
    rc = call_noalloc(body, arrays, tb.Settings(), capi.tl_step_report())
    assert rc == capi.TL_ERR_TOO_LARGE
    assert capi.lib().tl_status_string(rc) == b"input exceeds the fixed capacity of tl_step_noalloc"


@pytest.mark.gpu
def test_noalloc_step_honours_per_element_youngs_modulus():
    """A mesh with per-element Young's moduli steps like the resident system
    given the same moduli (and unlike the lane's own modulus)."""
    mesh, mat = elastic_block((6, 6, 6), seed=4)
    rng = np.random.default_rng(11)
    mesh.element_youngs = mat.youngs_modulus * np.exp(0.3 * rng.standard_normal(mesh.tets))
    settings = tb.Settings(law=tb.NEO_HOOKEAN)
    body = _Body(mesh, [mat])
    mine, ref = host_arrays(mesh), host_arrays(mesh)
    system = tb.System(mesh, [mat], tb.FP64)
    for call in range(2):
        assert call_noalloc(body, mine, settings, capi.tl_step_report()) == capi.TL_OK
        assert call_host(system, ref, settings, capi.tl_step_report()) == capi.TL_OK
        assert relative_error(mine["position"], ref["position"], mesh.rest_positions) <= 1e-9, call
    system.close()
    mesh.element_youngs = None
    lane_only = host_arrays(mesh)
    plain = _Body(mesh, [mat])
    for call in range(2):
        assert call_noalloc(plain, lane_only, settings, capi.tl_step_report()) == capi.TL_OK
    assert relative_error(lane_only["position"], ref["position"], mesh.rest_positions) > 1e-6


@pytest.mark.gpu
def test_noalloc_refuses_only_damping_an_element_uses():
    """An unused damped lane, or one with infinite damping (no damping), is
    accepted; a damped lane an element uses is refused before any work."""
    mesh, mat = elastic_block((4, 4, 4))
    damped = tb.PhysicalMaterial(density=1000.0, youngs_modulus=1e6, poissons_ratio=0.3, stiffness_damping=0.02)
    endless = tb.PhysicalMaterial(density=1000.0, youngs_modulus=1e6, poissons_ratio=0.3,
                                  stiffness_damping=float("inf"))
    for lanes, want in (([mat, damped], capi.TL_OK), ([endless], capi.TL_OK), ([damped], capi.TL_ERR_UNSUPPORTED)):
        arrays = host_arrays(mesh)
        rc = call_noalloc(_Body(mesh, lanes), arrays, tb.Settings(), capi.tl_step_report())
        assert rc == want, lanes
