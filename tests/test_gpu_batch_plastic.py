"""Yielding bodies in one batched system: the plastic Newton loop
(solver.cc:3951-4250) of every body at once.

Each yielding body runs its own Newton control (attempts, backtracking, the
linear-read hand-off, the fallback and its rejection) as a state machine; the
device work of all bodies is issued together in rounds, gated per body
(tl_system.cu: newtonBatch).  A ragged batch of plastic blocks pushed from
the top, with an elastic body among them, must give every body the result
and the Newton counts it gets alone (the plastic bar, 1e-8) and from the FP64
oracle.
"""
import numpy as np
import pytest

import talus_b200 as tb
from tests.helpers import GRAVITY, DT, plastic_block, relative_error, run_oracle

pytestmark = pytest.mark.gpu

CELLS = [(4, 4, 4), (6, 4, 5), (5, 8, 4), (4, 6, 6)]


def bodies():
    meshes, mats = [], []
    for k, cells in enumerate(CELLS):
        mesh, mat = plastic_block(cells=cells, seed=30 + k, speed=0.3 + 0.2 * k)
        meshes.append(mesh)
        mats.append([mat])
    elastic = tb.box_mesh((4, 5, 4), voxel=0.1, jitter=0.01, seed=40)
    meshes.insert(2, elastic)
    mats.insert(2, [tb.PhysicalMaterial(density=1000.0, youngs_modulus=1e6, poissons_ratio=0.3)])
    return meshes, mats


def step_batch(meshes, mats, precision, steps, settings):
    system = tb.System(meshes, mats, precision)
    for i, m in enumerate(meshes):
        system.set_state(tb.rest_state(m), i)
    counts = []
    for _ in range(steps):
        reps = system.step(settings, GRAVITY, DT)
        counts.append([(r.plastic_evaluations, r.plastic_solves, r.plastic_backtracks, r.cg_iterations)
                       for r in reps])
    states = [system.get_state(i) for i in range(len(meshes))]
    system.close()
    return states, counts


@pytest.mark.parametrize("form", ["assembled", "elementwise"])
def test_plastic_batch_equals_each_body_alone(form):
    meshes, mats = bodies()
    settings = tb.Settings()
    steps = 6
    system = tb.System(meshes, mats, tb.FP64)
    system.set_solver(form)
    for i, m in enumerate(meshes):
        system.set_state(tb.rest_state(m), i)
    batch_counts = []
    for _ in range(steps):
        reps = system.step(settings, GRAVITY, DT)
        batch_counts.append([(r.plastic_evaluations, r.plastic_solves, r.plastic_backtracks) for r in reps])
    batch = [system.get_state(i) for i in range(len(meshes))]
    system.close()
    for i, (m, mat) in enumerate(zip(meshes, mats)):
        alone = tb.System(m, mat, tb.FP64)
        alone.set_solver(form)
        alone.set_state(tb.rest_state(m))
        for k in range(steps):
            r = alone.step(settings, GRAVITY, DT)[0]
            assert (r.plastic_evaluations, r.plastic_solves, r.plastic_backtracks) == batch_counts[k][i], (i, k)
        got = alone.get_state()
        alone.close()
        # alone a body runs the single-body PCG kernels, in the batch the batched ones: the same
        # operator summed in another order, so the plastic path's FP64 bar applies
        assert relative_error(batch[i].position, got.position, m.rest_positions) <= 1e-8, i
        assert np.abs(batch[i].plastic[:, 9] - got.plastic[:, 9]).max() <= 1e-8 * max(1e-30, got.plastic[:, 9].max())
    evaluations = sum(c[i][0] for c in batch_counts for i in range(len(meshes)))
    assert evaluations > 3 * steps * len(CELLS)  # the Newton path ran


def test_plastic_batch_matches_the_oracle():
    meshes, mats = bodies()
    settings = tb.Settings()
    steps = 5
    states64, counts = step_batch(meshes, mats, tb.FP64, steps, settings)
    states32, _ = step_batch(meshes, mats, tb.FP32_MIXED, steps, settings)
    from oracle import pyoracle as po

    for i, (m, mat) in enumerate(zip(meshes, mats)):
        ostate, reports = run_oracle(po.F64, m, mat[0], settings, steps)
        assert relative_error(states64[i].position, ostate.position, m.rest_positions) <= 1e-8, i
        assert relative_error(states32[i].position, ostate.position, m.rest_positions) <= 1e-5, i
        assert [c[i][0] for c in counts] == [r["plastic_evaluations"] for r in reports], i
        if np.isfinite(mat[0].yield_stress):
            assert (ostate.plastic[:, 9] > 0).any(), i
