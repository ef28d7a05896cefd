"""The oracle against its committed golden fixtures (tests/golden/), CPU.

The fixtures were written by tests/golden/make_golden.py from the FP64
oracle; re-running the oracle must reproduce them, so a change to the
restatement of deformable::step (solver.cc:3472-4369, 5829-5900) or of the
tet laws (material.cc:236-265, 978-1057; neohookean.cc:41-90) shows here as a
changed number, not only as a GPU/oracle disagreement.  The fixtures also carry
properties any correct step has: pinned nodes sit at rest, element forces of a
tet sum to zero.
"""
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from tests.golden import make_golden as mg
from tests.helpers import DT, oracle_material, relative_error, run_oracle

GOLDEN = os.path.dirname(mg.__file__)


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


@pytest.mark.parametrize("name", sorted(mg.BLOCKS))
def test_generator_rebuilds_the_fixture_mesh(name):
    mesh, mat, settings, steps = mg.block_case(name)
    g = load(name)
    np.testing.assert_allclose(mg.mesh_checksum(mesh), g["mesh_checksum"], rtol=1e-12)
    np.testing.assert_array_equal(mg.material_array(mat), g["material"])
    assert int(g["law"]) == settings.law and int(g["steps"]) == steps


@pytest.mark.parametrize("name", sorted(mg.BLOCKS))
def test_oracle_reproduces_block_fixture(name):
    mesh, mat, settings, steps = mg.block_case(name)
    g = load(name)
    record = []
    state, reports = run_oracle(po.F64, mesh, mat, settings, steps, record=record)
    assert relative_error(record[0], g["first"], mesh.rest_positions) <= 1e-10
    assert relative_error(record[-1], g["last"], mesh.rest_positions) <= 1e-10
    assert [r["cg_iterations"] for r in reports] == list(g["cg_iterations"])
    assert [r["plastic_evaluations"] for r in reports] == list(g["plastic_evaluations"])
    np.testing.assert_allclose(state.plastic[:, 9], g["equivalent"], rtol=0, atol=1e-10)


@pytest.mark.parametrize("name", sorted(mg.BLOCKS))
def test_block_fixture_properties(name):
    mesh, mat, settings, steps = mg.block_case(name)
    g = load(name)
    pinned = mesh.anchored != 0
    # pinned nodes move only with their prescribed velocity (solver.cc:1035-1039)
    v = np.zeros((mesh.nodes, 3)) if mesh.prescribed_velocity is None else mesh.prescribed_velocity
    for x, n in ((g["first"], 1), (g["last"], steps)):
        np.testing.assert_allclose(x[pinned], mesh.rest_positions[pinned] + n * DT * v[pinned],
                                   rtol=0, atol=1e-12)
    assert np.isfinite(g["last"]).all() and np.isfinite(g["last_fp32"]).all()
    # the reference's own FP32 arithmetic stays near FP64 on these blocks
    assert relative_error(g["last_fp32"], g["last"], mesh.rest_positions) <= 1e-3
    if np.isfinite(mat.yield_stress):
        assert g["equivalent"].max() > 0.0 and (g["equivalent"] >= 0.0).all()
    else:
        assert not g["equivalent"].any()


def test_oracle_reproduces_the_single_tet_laws():
    g = load("tet_laws")
    el = oracle_material(mg.material_of(g["elastic"]))
    pl = oracle_material(mg.material_of(g["plastic"]))
    for e in range(g["rest"].shape[0]):
        args = (g["deformed"][e], g["rest"][e], g["rest_inverse"][e], g["volume"][e])
        scale = max(np.abs(g["corotated_force"][e]).max(), 1e-300)
        np.testing.assert_allclose(po.tet_trial(po.F64, *args, el)["force"], g["corotated_force"][e], rtol=0,
                                   atol=1e-12 * scale)
        scale = np.abs(g["snh_force"][e]).max()
        np.testing.assert_allclose(po.snh_tet(po.F64, *args, el)["force"], g["snh_force"][e], rtol=0,
                                   atol=1e-12 * scale)
        p = po.tet_point_trial(po.F64, *args, pl, tangent=False)
        scale = np.abs(g["plastic_force"][e]).max()
        np.testing.assert_allclose(p["force"], g["plastic_force"][e], rtol=0, atol=1e-12 * scale)
        np.testing.assert_allclose(p["plastic"], g["plastic_point"][e], rtol=0, atol=1e-14)
        assert p["yielding"] == g["yielding"][e]


def test_single_tet_fixture_properties():
    g = load("tet_laws")
    for key in ("corotated_force", "snh_force", "plastic_force"):
        f = g[key]
        # each element's corner forces balance (translation invariance of every law)
        assert np.abs(f.sum(axis=1)).max() <= 1e-9 * np.abs(f).max(), key
        assert np.isfinite(f).all(), key
    inverted = np.linalg.det(np.einsum("eij,ejk->eik", np.stack(
        [g["deformed"][:, k] - g["deformed"][:, 0] for k in (1, 2, 3)], axis=2), g["rest_inverse"])) <= 0.0
    assert inverted.sum() == 3
    # small deformations stay elastic, large ones yield
    assert g["yielding"][0::4].sum() == 0 and g["yielding"][3::4].all()


def test_oracle_reproduces_the_finite_strain_fixture():
    """hencky_block.npz: the plastic block in the finite-strain plasticity
    mode (plasticflow.cc:96-150, 184-247 at one point per tet)."""
    mesh, mat, settings, steps = mg.hencky_case()
    g = load("hencky_block")
    np.testing.assert_allclose(mg.mesh_checksum(mesh), g["mesh_checksum"], rtol=1e-12)
    record = []
    state, reports = run_oracle(po.F64, mesh, mat, settings, steps, record=record, plasticity=po.PLASTICITY_HENCKY)
    assert relative_error(record[0], g["first"], mesh.rest_positions) <= 1e-10
    assert relative_error(record[-1], g["last"], mesh.rest_positions) <= 1e-10
    assert [r["yielding"] for r in reports] == list(g["flowed"])
    assert [r["cg_iterations"] for r in reports] == list(g["cg_iterations"])
    np.testing.assert_allclose(state.plastic[:, 9], g["hardening"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(state.plastic[::mg.HENCKY_SAMPLE, :9], g["plastic_map_sample"], rtol=0, atol=1e-12)
    # the flow is deviatoric: every stored plastic map keeps volume
    maps = g["plastic_map_sample"].reshape(-1, 3, 3)
    assert np.abs(np.linalg.det(maps) - 1.0).max() <= 1e-12
