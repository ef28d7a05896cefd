"""Floating bodies on the GPU against the oracle, through the C ABI.

A body with no anchored node, stepped with the rigid split on (floats,
solver.cc:2964-2971), runs in the frame of its centre and rigid spin
(floatingFrame solver.cc:3031-3142, predictor and drive solver.cc:3657-3690,
return to the world and momentum projection solver.cc:4265-4340).  Bars: FP64
within 1e-9 relative displacement of the FP64 oracle with the same PCG
iteration counts, FP32-mixed within 1e-5.
"""
import numpy as np
import pytest

import talus_b200 as tb
from talus_b200 import _capi as capi
from oracle import pyoracle as po
from tests.helpers import DT, GRAVITY, oracle_material, oracle_settings, relative_error, to_oracle

pytestmark = pytest.mark.gpu

SPLITS = {"projected": capi.TL_RIGID_SPLIT_PROJECTED, "unprojected": capi.TL_RIGID_SPLIT_UNPROJECTED}


def floating_block(cells=(8, 8, 8), seed=7):
    mesh = tb.box_mesh(cells, voxel=0.1, jitter=0.01, seed=seed, anchor_axis=3)
    assert mesh.anchored.sum() == 0
    return mesh


def spun(mesh, omega=(0.4, 3.0, 1.0), drift=(0.5, 1.0, 0.0)):
    """Rest state with a rigid spin about the centre and a drift."""
    state = tb.rest_state(mesh)
    m = mesh.node_mass[:, None]
    centre = (m * mesh.rest_positions).sum(0) / m.sum()
    state.velocity[...] = np.cross(np.asarray(omega, float), mesh.rest_positions - centre) + np.asarray(drift)
    return state


def run_both(precision, mesh, mat, settings, steps, state0):
    om = to_oracle(mesh)
    ostate = po.State(state0.position.copy(), state0.velocity.copy(), state0.acceleration.copy(),
                      state0.rotation.copy(), state0.plastic.copy())
    system = tb.System(mesh, [mat], precision)
    system.set_state(state0)
    worst, iters = 0.0, []
    for _ in range(steps):
        rep = po.step(po.F64, om, ostate, [oracle_material(mat)], oracle_settings(settings), GRAVITY, DT)
        grep = system.step(settings, GRAVITY, DT)[0]
        got = system.get_state()
        worst = max(worst, relative_error(got.position, ostate.position, mesh.rest_positions))
        iters.append((rep.cg_iterations, grep.cg_iterations, rep.plastic_evaluations, grep.plastic_evaluations))
    final = system.get_state()
    system.close()
    return worst, iters, final, ostate


@pytest.mark.parametrize("law", [tb.COROTATED, tb.NEO_HOOKEAN])
@pytest.mark.parametrize("split", sorted(SPLITS))
def test_spinning_free_body_fp64_matches_the_oracle(law, split):
    mesh = floating_block()
    mat = tb.PhysicalMaterial(density=1000.0, youngs_modulus=1e6, poissons_ratio=0.3)
    settings = tb.Settings(law=law, rigid_split=SPLITS[split])
    worst, iters, got, want = run_both(tb.FP64, mesh, mat, settings, 10, spun(mesh))
    assert worst <= 1e-9, worst
    for o_it, g_it, _, _ in iters:
        assert o_it == g_it
    assert np.abs(got.velocity - want.velocity).max() <= 1e-9 * np.abs(want.velocity).max()
    if law == tb.COROTATED:  # committed rotations turn with the frame (solver.cc:4343-4345)
        assert np.abs(got.rotation - want.rotation).max() <= 1e-8


@pytest.mark.parametrize("split", sorted(SPLITS))
def test_spinning_free_body_fp32_mixed_within_1e5(split):
    mesh = floating_block()
    mat = tb.PhysicalMaterial(density=1000.0, youngs_modulus=1e6, poissons_ratio=0.3)
    settings = tb.Settings(law=tb.NEO_HOOKEAN, rigid_split=SPLITS[split])
    worst, _, _, _ = run_both(tb.FP32_MIXED, mesh, mat, settings, 10, spun(mesh))
    assert worst <= 1e-5, worst


def test_free_fall_is_a_rigid_translation():
    mesh = floating_block((6, 4, 5))
    mat = tb.PhysicalMaterial(density=1000.0, youngs_modulus=1e6, poissons_ratio=0.3)
    system = tb.System(mesh, [mat], tb.FP64)
    system.set_state(tb.rest_state(mesh))
    for _ in range(12):
        system.step(tb.Settings(), GRAVITY, DT)
    moved = system.get_state().position - mesh.rest_positions
    mean = moved.mean(0)
    assert np.abs(moved - mean).max() <= 1e-9 * np.abs(mean).max()
    system.close()


def test_plastic_spinning_body_takes_the_newton_path_like_the_oracle():
    """Centrifugal stress past a low yield stress: the plastic Newton loop in
    the frame, with the same Newton evaluation counts as the oracle."""
    mesh = floating_block((6, 4, 4), seed=9)
    mat = tb.PhysicalMaterial(density=1000.0, youngs_modulus=1e6, poissons_ratio=0.3, yield_stress=1.5e3,
                              hardening_modulus=1e4)
    settings = tb.Settings(rigid_split=SPLITS["projected"])
    worst, iters, got, want = run_both(tb.FP64, mesh, mat, settings, 6, spun(mesh, omega=(0.0, 9.0, 2.0)))
    assert worst <= 1e-8, worst
    assert sum(i[2] for i in iters) > 6  # the Newton path ran
    for o_it, g_it, o_ev, g_ev in iters:
        assert o_ev == g_ev
    assert (want.plastic[:, 9] > 0).any()
    assert np.abs(got.plastic[:, 9] - want.plastic[:, 9]).max() <= 1e-8 * want.plastic[:, 9].max()


@pytest.mark.parametrize("graph", [False, True])
def test_batch_of_anchored_and_floating_bodies_equals_each_alone(graph):
    meshes = [floating_block((3, 4, 2), seed=11), tb.box_mesh((4, 3, 3), voxel=0.1, jitter=0.01, seed=12),
              floating_block((2, 2, 5), seed=13)]
    mats = [[tb.PhysicalMaterial(density=1000.0, youngs_modulus=e, poissons_ratio=0.3)] for e in (1e6, 3e6, 5e5)]
    starts = [spun(meshes[0]), tb.rest_state(meshes[1]), spun(meshes[2], omega=(2.0, 0.0, 1.0))]
    settings = tb.Settings(law=tb.NEO_HOOKEAN)
    batch = tb.System(meshes, mats, tb.FP64)
    batch.tune(0, graph)
    for i, s in enumerate(starts):
        batch.set_state(s, i)
    for _ in range(6):
        batch.step(settings, GRAVITY, DT)
    for i, (m, mat, s) in enumerate(zip(meshes, mats, starts)):
        alone = tb.System(m, mat, tb.FP64)
        alone.set_state(s)
        for _ in range(6):
            alone.step(settings, GRAVITY, DT)
        assert relative_error(batch.get_state(i).position, alone.get_state().position, m.rest_positions) <= 1e-10
        alone.close()
    batch.close()


def test_rigid_split_off_steps_an_unanchored_body_on_the_ordinary_path():
    mesh = floating_block((4, 4, 4))
    mat = tb.PhysicalMaterial(density=1000.0, youngs_modulus=1e6, poissons_ratio=0.3)
    settings = tb.Settings(rigid_split=capi.TL_RIGID_SPLIT_OFF)
    worst, iters, _, _ = run_both(tb.FP64, mesh, mat, settings, 5, spun(mesh))
    assert worst <= 1e-9
