"""The CUDA path against the committed golden fixtures (tests/golden/).

No CPU solve runs here: every expected value comes from a fixture the FP64
oracle wrote (tests/golden/make_golden.py).  Bars as in test_gpu_parity:
FP64 <= 1e-9 relative displacement error on the elastic and damped blocks and
1e-8 on the plastic Newton path, FP32-mixed <= 1e-5 (the FP32-mixed
tolerance); each solver form (element-wise, assembled) meets them.  Single
tets: element forces of each law through tl_evaluate, FP64 within 1e-9 of the
tet's largest corner force and FP32-mixed within 1e-4 (the force tolerance of
test_gpu_inversion), yield flags exact in FP64.
"""
import os

import numpy as np
import pytest

import talus_b200 as tb
from tests.golden import make_golden as mg
from tests.helpers import DT, GRAVITY, relative_error

pytestmark = pytest.mark.gpu

GOLDEN = os.path.dirname(mg.__file__)


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


@pytest.mark.parametrize("form", ["elementwise", "assembled"])
@pytest.mark.parametrize("name", sorted(mg.BLOCKS))
@pytest.mark.parametrize("precision", [tb.FP64, tb.FP32_MIXED], ids=["fp64", "mixed"])
def test_block_matches_golden(name, precision, form):
    mesh, mat, settings, steps = mg.block_case(name)
    g = load(name)
    np.testing.assert_allclose(mg.mesh_checksum(mesh), g["mesh_checksum"], rtol=1e-12)
    plastic = np.isfinite(mat.yield_stress)
    tol = 1e-5 if precision == tb.FP32_MIXED else (1e-8 if plastic else 1e-9)
    system = tb.System(mesh, [mat], precision)
    system.set_solver(form)
    system.set_state(tb.rest_state(mesh))
    reports = []
    first = None
    for i in range(steps):
        reports.append(system.step(settings, GRAVITY, DT)[0].as_dict())
        if i == 0:
            first = system.get_state().position
    state = system.get_state()
    system.close()
    assert relative_error(first, g["first"], mesh.rest_positions) <= tol
    assert relative_error(state.position, g["last"], mesh.rest_positions) <= tol
    if precision == tb.FP64:
        assert [r["plastic_evaluations"] for r in reports] == list(g["plastic_evaluations"])
        scale = max(1.0, np.abs(g["equivalent"]).max())
        assert np.abs(state.plastic[:, 9] - g["equivalent"]).max() <= 1e-8 * scale


def single_tet_system(g, mat, precision):
    count = g["rest"].shape[0]
    volume = g["volume"]
    mesh = tb.PreparedMesh(
        rest_positions=g["rest"].reshape(-1, 3).copy(), node_mass=np.repeat(mat.density * volume / 4.0, 4),
        anchored=np.zeros(4 * count, np.uint8), tet_nodes=np.arange(4 * count, dtype=np.uint32).reshape(count, 4),
        rest_inverse=g["rest_inverse"].copy(), volume=volume.copy(), material=np.zeros(count, np.uint32))
    system = tb.System(mesh, [mat], precision)
    state = tb.rest_state(mesh)
    state.position = g["deformed"].reshape(-1, 3).copy()
    system.set_state(state)
    return system


@pytest.mark.parametrize("precision", [tb.FP64, tb.FP32_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("law,material,key", [(tb.COROTATED, "elastic", "corotated_force"),
                                              (tb.NEO_HOOKEAN, "elastic", "snh_force"),
                                              (tb.COROTATED, "plastic", "plastic_force")],
                         ids=["corotated", "snh", "plastic"])
def test_single_tet_forces_match_golden(law, material, key, precision):
    g = load("tet_laws")
    system = single_tet_system(g, mg.material_of(g[material]), precision)
    forces, yielding = system.evaluate(tb.Settings(law=law))
    system.close()
    forces = forces.reshape(-1, 4, 3)
    expected = g[key]
    scale = np.abs(expected).max(axis=(1, 2), keepdims=True)
    worst = float((np.abs(forces - expected) / scale).max())
    assert worst <= (1e-9 if precision == tb.FP64 else 1e-4), worst
    if material == "plastic" and precision == tb.FP64:
        np.testing.assert_array_equal(yielding, g["yielding"])


@pytest.mark.parametrize("form", ["elementwise", "assembled"])
@pytest.mark.parametrize("precision", [tb.FP64, tb.FP32_MIXED], ids=["fp64", "mixed"])
def test_finite_strain_block_matches_golden(precision, form):
    mesh, mat, settings, steps = mg.hencky_case()
    g = load("hencky_block")
    np.testing.assert_allclose(mg.mesh_checksum(mesh), g["mesh_checksum"], rtol=1e-12)
    system = tb.System(mesh, [mat], precision)
    system.set_solver(form)
    system.set_plasticity("hencky")
    system.set_state(tb.rest_state(mesh, hencky=True))
    tol = 1e-9 if precision == tb.FP64 else 1e-5
    flowed, first = [], None
    for i in range(steps):
        flowed.append(system.step(settings, GRAVITY, DT)[0].yielding)
        if i == 0:
            first = system.get_state().position
    state = system.get_state()
    system.close()
    assert relative_error(first, g["first"], mesh.rest_positions) <= tol
    assert relative_error(state.position, g["last"], mesh.rest_positions) <= tol
    if precision == tb.FP64:
        assert flowed == list(g["flowed"])
        assert np.abs(state.plastic[:, 9] - g["hardening"]).max() <= 1e-9 * max(1.0, g["hardening"].max())
        assert np.abs(state.plastic[::mg.HENCKY_SAMPLE, :9] - g["plastic_map_sample"]).max() <= 1e-9
