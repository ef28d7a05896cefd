"""The oracle's floating-body frame (CPU, no GPU).

A body with no anchored node and RigidSplit on (floats, solver.cc:2964-2971)
is stepped in a frame that moves with its centre of mass and turns with its
rigid spin (floatingFrame solver.cc:3031-3142, the predictor and drive
solver.cc:3657-3690, the return to the world and the momentum projection
solver.cc:4265-4340).  The reference has no test of this path; these tests
pin the restatement on what the equations must give:

* free fall of an unstressed body is a rigid translation whose centre follows
  the generalized-alpha recurrence of constant gravity, the same as with
  RigidSplit::Off;
* a rigidly spinning body without gravity keeps its linear momentum at zero
  and, with the Projected split, its angular momentum (the projection restores
  the frame's rigid momentum every substep);
* the FP32 oracle (the reference's own arithmetic) follows the FP64 oracle.
"""
import math

import numpy as np
import pytest

import talus_b200 as tb
from oracle import pyoracle as po
from tests.helpers import DT, to_oracle

RUBBER = po.material(1000.0, 1e6, 0.3)


def floating_block(cells=(4, 4, 4), jitter=0.0, seed=5):
    mesh = tb.box_mesh(cells, voxel=0.1, jitter=jitter, seed=seed, anchor_axis=3)
    assert mesh.anchored.sum() == 0
    return to_oracle(mesh)


def generalized_alpha_fall(g, steps, dt=DT, spectral=0.5):
    """Centre of a body under constant gravity, integrated by the frame's own
    recurrence: next = (g - am a) / (1 - am), c += h v + h^2 ((1/2 - b) a + b next),
    v += h ((1 - gm) a + gm next), a = next."""
    rho = spectral
    am, af = (2 * rho - 1) / (rho + 1), rho / (rho + 1)
    gm, b = 0.5 - am + af, 0.25 * (1 - am + af) ** 2
    c = np.zeros(3)
    v = np.zeros(3)
    a = np.zeros(3)
    g = np.asarray(g, float)
    for _ in range(steps):
        nxt = (g - am * a) / (1 - am)
        c = c + dt * v + dt * dt * ((0.5 - b) * a + b * nxt)
        v = v + dt * ((1 - gm) * a + gm * nxt)
        a = nxt
    return c, v


def momenta(mesh, state):
    m = mesh.node_mass[:, None]
    centre = (m * state.position).sum(0) / m.sum()
    linear = (m * state.velocity).sum(0)
    angular = (m * np.cross(state.position - centre, state.velocity)).sum(0)
    return linear, angular


@pytest.mark.parametrize("split", [po_split for po_split in (1, 2)])
def test_free_fall_is_a_rigid_translation_on_the_frame_recurrence(split):
    mesh = floating_block()
    state = po.State.rest(mesh)
    g = (0.0, -9.81, 0.0)
    steps = 12
    for _ in range(steps):
        po.step(po.F64, mesh, state, [RUBBER], po.Settings(rigid_split=split), g, DT)
    moved = state.position - mesh.rest
    centre, velocity = generalized_alpha_fall(g, steps)
    assert np.abs(moved - centre).max() <= 1e-9 * np.abs(centre).max()
    assert np.abs(state.velocity - velocity).max() <= 1e-9 * np.abs(velocity).max()


def test_free_fall_floating_equals_the_ordinary_path():
    mesh = floating_block(jitter=0.01)
    runs = []
    for split in (0, 2):
        state = po.State.rest(mesh)
        for _ in range(8):
            po.step(po.F64, mesh, state, [RUBBER], po.Settings(rigid_split=split), (0.0, -9.81, 0.0), DT)
        runs.append(state.position - mesh.rest)
    scale = np.abs(runs[1]).max()
    assert np.abs(runs[0] - runs[1]).max() <= 1e-8 * scale


def spinning_state(mesh, omega=(0.0, 2.0, 1.0), drift=(0.3, 0.0, 0.0)):
    state = po.State.rest(mesh)
    m = mesh.node_mass[:, None]
    centre = (m * mesh.rest).sum(0) / m.sum()
    state.velocity[...] = np.cross(np.asarray(omega, float), mesh.rest - centre) + np.asarray(drift)
    return state


def test_projected_split_keeps_linear_and_angular_momentum_of_a_spinning_body():
    mesh = floating_block(cells=(4, 3, 2), jitter=0.01)
    state = spinning_state(mesh)
    linear0, angular0 = momenta(mesh, state)
    for _ in range(20):
        po.step(po.F64, mesh, state, [RUBBER], po.Settings(rigid_split=2), (0.0, 0.0, 0.0), DT)
    linear, angular = momenta(mesh, state)
    assert np.abs(linear - linear0).max() <= 1e-9 * np.abs(linear0).max()
    assert np.abs(angular - angular0).max() <= 1e-7 * np.abs(angular0).max()
    # the body turned rigidly: distances to the centre are kept to the elastic strain
    m = mesh.node_mass[:, None]
    arm0 = mesh.rest - (m * mesh.rest).sum(0) / m.sum()
    arm = state.position - (m * state.position).sum(0) / m.sum()
    assert np.abs(np.linalg.norm(arm, axis=1) - np.linalg.norm(arm0, axis=1)).max() < 2e-3 * 0.3
    # and it turned by the spin's angle about its axis (|omega| t)
    turned = math.acos(np.clip(np.dot(arm0[0], arm[0]) / np.linalg.norm(arm0[0]) / np.linalg.norm(arm[0]), -1, 1))
    assert turned > 0.1


def test_unprojected_split_runs_and_differs_from_projected():
    mesh = floating_block(cells=(4, 3, 2), jitter=0.01)
    ends = []
    for split in (1, 2):
        state = spinning_state(mesh)
        for _ in range(10):
            po.step(po.F64, mesh, state, [RUBBER], po.Settings(rigid_split=split), (0.0, -9.81, 0.0), DT)
        assert np.isfinite(state.position).all()
        ends.append(state.position.copy())
    scale = np.abs(ends[1] - mesh.rest).max()
    gap = np.abs(ends[0] - ends[1]).max()
    assert 0.0 < gap < 1e-2 * scale


def test_fp32_oracle_follows_fp64_on_a_spinning_body():
    mesh = floating_block(cells=(4, 3, 2), jitter=0.01)
    ends = []
    for precision in (po.F64, po.F32):
        state = spinning_state(mesh)
        for _ in range(10):
            po.step(precision, mesh, state, [RUBBER], po.Settings(rigid_split=2), (0.0, -9.81, 0.0), DT)
        ends.append(state.position.copy())
    scale = np.linalg.norm(ends[0] - mesh.rest, axis=1).max()
    assert np.linalg.norm(ends[1] - ends[0], axis=1).max() <= 1e-3 * scale
