"""Invalid inputs come back as TL_ERR_ARG before anything reaches a device.

The reference steps only meshes its buildMesh made: tets of positive volume
(solver.cc:2352-2356), nullptr for an invalid lattice (solver.cc:2193-2198,
2405-2407).  A caller-built tl_mesh_desc is held to the same rules: finite
rest positions, rest inverses and prescribed velocities, volumes > 0, masses
>= 0, node indices in range, material lanes with a finite E >= 0.  tl_step
also wants a finite dt > 0 and finite gravity.  tl_step_noalloc checks all of
this before it looks for a device, so these cases run on the CPU; the resident
system's creation applies the same checks (GPU case at the end).
"""
import ctypes as C
import math

import numpy as np
import pytest

import talus_b200 as tb
from talus_b200 import _capi as capi
from talus_b200.deformable import _Body
from tests.helpers import DT, GRAVITY, elastic_block


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def noalloc(mesh, mat, dt=DT, gravity=GRAVITY):
    body = _Body(mesh, [mat])
    s = tb.rest_state(mesh)
    arrays = [np.ascontiguousarray(getattr(s, k), np.float64) for k in
              ("position", "velocity", "acceleration", "rotation", "plastic")]
    g = np.asarray(gravity, np.float64)
    report = capi.tl_step_report()
    return capi.lib().tl_step_noalloc(0, C.byref(body.desc), capi.TL_DTYPE_F64, *[a.ctypes.data for a in arrays],
                                      C.byref(tb.Settings()._c()), g.ctypes.data, dt, C.byref(report))


def small():
    return elastic_block((3, 3, 3), seed=5)


def spoil(what):
    mesh, mat = small()
    if what == "rest_nan":
        mesh.rest_positions[7, 1] = math.nan
    elif what == "rest_inverse_inf":
        mesh.rest_inverse[3, 2, 0] = math.inf
    elif what == "zero_volume":
        mesh.volume[11] = 0.0
    elif what == "negative_mass":
        mesh.node_mass[2] = -1.0
    elif what == "node_out_of_range":
        mesh.tet_nodes[5, 3] = mesh.nodes
    elif what == "element_youngs_zero":
        mesh.element_youngs = np.full(mesh.tets, 1e6)
        mesh.element_youngs[4] = 0.0
    elif what == "prescribed_nan":
        mesh.prescribed_velocity = np.zeros((mesh.nodes, 3))
        mesh.prescribed_velocity[np.flatnonzero(mesh.anchored)[0], 0] = math.nan
    elif what == "negative_youngs":
        mat.youngs_modulus = -1.0
    elif what == "nan_hardening":
        mat.yield_stress, mat.hardening_modulus = 1e5, math.nan
    return mesh, mat


SPOILS = ["rest_nan", "rest_inverse_inf", "zero_volume", "negative_mass", "node_out_of_range",
          "element_youngs_zero", "prescribed_nan", "negative_youngs", "nan_hardening"]


@pytest.mark.parametrize("what", SPOILS)
def test_invalid_mesh_is_refused_before_any_device_work(what):
    mesh, mat = spoil(what)
    assert noalloc(mesh, mat) == capi.TL_ERR_ARG


@pytest.mark.parametrize("dt,gravity", [(math.inf, GRAVITY), (math.nan, GRAVITY), (0.0, GRAVITY), (-DT, GRAVITY),
                                        (DT, (0.0, math.nan, 0.0)), (DT, (math.inf, 0.0, 0.0))])
def test_invalid_step_arguments_are_refused(dt, gravity):
    mesh, mat = small()
    assert noalloc(mesh, mat, dt=dt, gravity=gravity) == capi.TL_ERR_ARG


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_valid_mesh_passes_the_checks_and_then_needs_a_device():
    mesh, mat = small()
    assert noalloc(mesh, mat) == capi.TL_ERR_NO_DEVICE
    # an infinite yield stress with any hardening is elastic, and E = 0 is the reference's default lane
    mat.hardening_modulus = math.nan
    mat.youngs_modulus = 0.0
    assert noalloc(mesh, mat) == capi.TL_ERR_NO_DEVICE


@pytest.mark.gpu
@pytest.mark.parametrize("what", SPOILS)
def test_system_creation_refuses_invalid_meshes(what):
    mesh, mat = spoil(what)
    with pytest.raises(capi.TalusError) as err:
        tb.System(mesh, [mat], tb.FP64)
    assert err.value.status == capi.TL_ERR_ARG
