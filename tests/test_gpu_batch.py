"""Batched systems and determinism of the CUDA step.

* A system holding several bodies steps each body exactly as a system holding
  that body alone (the batched form shares launches, not physics).
* Two runs of the same inputs give bitwise-identical states: every
  reduction is in a fixed order and the assembly is a gather, with no
  floating-point atomics (the reference's run-to-run determinism,
  tests/dynamics_strainstep_tests.cc:4998-5050).
"""
import numpy as np
import pytest

import talus_b200 as tb
from tests.helpers import DT, GRAVITY, elastic_block, plastic_block

pytestmark = pytest.mark.gpu


def bodies():
    a, ma = elastic_block((6, 5, 4), seed=3)
    b, mb = elastic_block((3, 7, 5), seed=4)
    mb = tb.PhysicalMaterial(density=800.0, youngs_modulus=3e5, poissons_ratio=0.42)
    c, mc = elastic_block((9, 4, 3), seed=5)
    mc = tb.PhysicalMaterial(density=1200.0, youngs_modulus=5e6, poissons_ratio=0.28)
    return [a, b, c], [[ma], [mb], [mc]]


@pytest.mark.parametrize("law", [tb.COROTATED, tb.NEO_HOOKEAN])
@pytest.mark.parametrize("precision,tol", [(tb.FP64, 1e-10), (tb.FP32_MIXED, 1e-5)])
def test_batched_bodies_match_single_body_systems(law, precision, tol):
    meshes, mats = bodies()
    settings = tb.Settings(law=law)
    batch = tb.System(meshes, mats, precision)
    for i, m in enumerate(meshes):
        batch.set_state(tb.rest_state(m), i)
    singles = []
    for m, mat in zip(meshes, mats):
        s = tb.System(m, mat, precision)
        s.set_state(tb.rest_state(m))
        singles.append(s)
    for _ in range(8):
        reports = batch.step(settings, GRAVITY, DT)
        for i, s in enumerate(singles):
            rep = s.step(settings, GRAVITY, DT)[0]
            assert reports[i].cg_iterations == rep.cg_iterations or precision == tb.FP32_MIXED
    for i, (m, s) in enumerate(zip(meshes, singles)):
        x = batch.get_state(i).position
        ref = s.get_state().position
        scale = np.linalg.norm(ref - m.rest_positions, axis=1).max()
        assert np.linalg.norm(x - ref, axis=1).max() <= tol * scale, i


@pytest.mark.parametrize("precision", [tb.FP64, tb.FP32_MIXED])
def test_runs_are_bitwise_identical(precision):
    mesh, mat = plastic_block()
    results = []
    for _ in range(2):
        s = tb.System(mesh, [mat], precision)
        s.set_state(tb.rest_state(mesh))
        for _ in range(6):
            s.step(tb.Settings(), GRAVITY, DT)
        st = s.get_state()
        results.append(np.concatenate([st.position.ravel(), st.velocity.ravel(), st.plastic.ravel()]))
        s.close()
    assert np.array_equal(results[0], results[1])


def test_host_state_step_matches_resident_step():
    """tl_step_host (the reference's calling convention, state in host memory)
    equals set/step/get on a resident system.  Positions cross the boundary as
    x = X + u, so each round trip may move them by an ulp."""
    mesh, mat = elastic_block()
    state = tb.rest_state(mesh)
    resident = tb.System(mesh, [mat], tb.FP64)
    resident.set_state(state)
    for _ in range(5):
        tb.step(mesh, state, [mat], tb.Settings(), GRAVITY, DT, precision=tb.FP64)
        resident.step(tb.Settings(), GRAVITY, DT)
    ref = resident.get_state().position
    scale = np.linalg.norm(ref - mesh.rest_positions, axis=1).max()
    assert np.linalg.norm(state.position - ref, axis=1).max() <= 1e-12 * scale
