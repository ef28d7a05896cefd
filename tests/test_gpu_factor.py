"""The caller-held solver state (DeformableSolverState, factor.h:205-210):
the FP64 Cholesky preconditioner, its refresh rules and its counters
(solver.cc:3606-3655, 3808-3910, 4258-4263), GPU (kPcgFactor, through the C
ABI) against the oracle with the same solver state.

Bars as in the other parity tests: FP64 <= 1e-9 relative displacement error
per step with the same PCG iteration count per step (elastic; 1e-8 with
yielding), FP32-mixed <= 1e-5 of FP64.  The factor's own ordering differs
from the oracle's (nested dissection against the oracle's envelope), so the
two preconditioners agree to rounding, not bitwise.
"""
import numpy as np
import pytest

import talus_b200 as tb
from oracle import pyoracle as po
from talus_b200 import _capi as capi
from tests.helpers import (DT, GRAVITY, elastic_block, oracle_material, oracle_settings, plastic_block,
                           relative_error, to_oracle)

pytestmark = pytest.mark.gpu

# counters the two must agree on exactly
COUNTERS = ("refactor_count", "retry_count", "substeps_since_refresh", "refresh_requested", "fresh_retry_failed",
            "rows", "ready", "system_nonzeros", "generation", "refresh_requests", "refactors", "retries",
            "retries_failed", "wasted_iterations", "spent_before_refresh", "spent_after_refresh", "refreshed_at_age",
            "factor_applications")


def run_factored(precision, mesh, mat, settings, steps, budget, state0=None, oracle=True):
    """Steps the GPU and (with oracle) the FP64 oracle, each with its own
    solver state; per-step errors, reports and both solver states' stats."""
    om = to_oracle(mesh)
    state0 = state0 if state0 is not None else tb.rest_state(mesh)
    ostate = po.State(state0.position.copy(), state0.velocity.copy(), state0.acceleration.copy(),
                      state0.rotation.copy(), state0.plastic.copy())
    osolver = po.Solver(budget)
    system = tb.System(mesh, [mat], precision)
    system.set_solver("assembled")
    system.use_factor(True, budget)
    system.set_state(state0)
    errors, greps, oreps, positions = [], [], [], []
    for _ in range(steps):
        if oracle:
            oreps.append(po.step(po.F64, om, ostate, [oracle_material(mat)], oracle_settings(settings), GRAVITY, DT,
                                 solver=osolver).as_dict())
        greps.append(system.step(settings, GRAVITY, DT)[0].as_dict())
        got = system.get_state()
        positions.append(got.position)
        if oracle:
            errors.append(relative_error(got.position, ostate.position, mesh.rest_positions))
    gstats = system.factor_stats()
    system.close()
    return errors, greps, oreps, gstats, osolver.stats(), positions


def assert_same_counters(gstats, ostats):
    for k in COUNTERS:
        assert gstats[k] == ostats[k], (k, gstats[k], ostats[k])
    assert abs(gstats["mean_iterations"] - ostats["mean_iterations"]) <= 1e-4 * max(1.0, ostats["mean_iterations"])


def test_factored_elastic_block_fp64_matches_oracle():
    mesh, mat = elastic_block()
    errors, greps, oreps, gstats, ostats, _ = run_factored(tb.FP64, mesh, mat, tb.Settings(), 6, budget=32)
    assert max(errors) <= 1e-9, errors
    assert [r["cg_iterations"] for r in greps] == [r["cg_iterations"] for r in oreps]
    assert_same_counters(gstats, ostats)
    assert gstats["ready"] == 1 and gstats["refactor_count"] == 1 and gstats["factor_nonzeros"] > 0
    # the factor conditions far better than block Jacobi
    assert max(r["cg_iterations"] for r in greps) < 20


def test_factored_step_solves_what_the_jacobi_step_solves():
    """Same equations, different preconditioner: the two trajectories agree
    to the PCG tolerance."""
    mesh, mat = elastic_block()
    settings = tb.Settings(tolerance=1e-8, cg_iterations=400)
    _, _, _, _, _, fact = run_factored(tb.FP64, mesh, mat, settings, 4, budget=32, oracle=False)
    system = tb.System(mesh, [mat], tb.FP64)
    system.set_solver("assembled")
    system.set_state(tb.rest_state(mesh))
    for x in fact:
        system.step(settings, GRAVITY, DT)
        assert relative_error(system.get_state().position, x, mesh.rest_positions) <= 1e-6
    system.close()


def test_factored_plastic_block_with_refreshes_fp64_matches_oracle():
    """A budget of 2 iterations caps the factored solves of a yielding block:
    every capped first solve refreshes the factor and solves again, and the
    counters of the refreshes follow the oracle's."""
    mesh, mat = plastic_block((8, 4, 4))
    errors, greps, oreps, gstats, ostats, _ = run_factored(tb.FP64, mesh, mat, tb.Settings(), 4, budget=2)
    assert max(errors) <= 1e-8, errors
    assert [r["cg_iterations"] for r in greps] == [r["cg_iterations"] for r in oreps]
    assert [r["plastic_evaluations"] for r in greps] == [r["plastic_evaluations"] for r in oreps]
    assert_same_counters(gstats, ostats)
    assert gstats["retries"] > 0 and gstats["wasted_iterations"] > 0


def test_factored_damped_block_fp64_matches_oracle():
    """Stiffness damping: the factor holds the damping blocks at the state's
    positions (factor.cc:346-366), refreshed with the damping scale."""
    mesh, _ = elastic_block()
    mat = tb.PhysicalMaterial(density=1000.0, youngs_modulus=1e6, poissons_ratio=0.3, stiffness_damping=0.02)
    errors, greps, oreps, gstats, ostats, _ = run_factored(tb.FP64, mesh, mat, tb.Settings(), 6, budget=32)
    assert max(errors) <= 1e-9, errors
    assert [r["cg_iterations"] for r in greps] == [r["cg_iterations"] for r in oreps]
    assert_same_counters(gstats, ostats)


def test_factored_spinning_free_body_fp64_matches_oracle():
    """A floating body: the factor is applied in the body's rotation since
    the refresh (bodyRotation)."""
    mesh = tb.box_mesh((6, 6, 6), voxel=0.1, jitter=0.01, seed=7, anchor_axis=3)
    mat = tb.PhysicalMaterial(density=1000.0, youngs_modulus=1e6, poissons_ratio=0.3)
    state = tb.rest_state(mesh)
    m = mesh.node_mass[:, None]
    centre = (m * mesh.rest_positions).sum(0) / m.sum()
    state.velocity[...] = np.cross(np.array([0.4, 3.0, 1.0]), mesh.rest_positions - centre)
    settings = tb.Settings(rigid_split=capi.TL_RIGID_SPLIT_PROJECTED)
    errors, greps, oreps, gstats, ostats, _ = run_factored(tb.FP64, mesh, mat, settings, 6, budget=32, state0=state)
    assert max(errors) <= 1e-9, errors
    assert [r["cg_iterations"] for r in greps] == [r["cg_iterations"] for r in oreps]
    assert_same_counters(gstats, ostats)


def test_factored_mixed_follows_fp64():
    mesh, mat = plastic_block((8, 4, 4))
    _, _, _, _, _, x64 = run_factored(tb.FP64, mesh, mat, tb.Settings(), 4, budget=32, oracle=False)
    _, _, _, _, _, x32 = run_factored(tb.FP32_MIXED, mesh, mat, tb.Settings(), 4, budget=32, oracle=False)
    worst = max(relative_error(a, b, mesh.rest_positions) for a, b in zip(x32, x64))
    assert worst <= 1e-5, worst


def test_step_change_refreshes_the_factor():
    """A new dt changes h: the next step makes the factor again (the
    reference compares FactorReference::step)."""
    mesh, mat = elastic_block((4, 4, 4))
    system = tb.System(mesh, [mat], tb.FP64)
    system.use_factor(True, 32)
    system.set_state(tb.rest_state(mesh))
    system.step(tb.Settings(), GRAVITY, DT)
    system.step(tb.Settings(), GRAVITY, DT)
    assert system.factor_stats()["refactor_count"] == 1
    system.step(tb.Settings(), GRAVITY, DT / 2)
    assert system.factor_stats()["refactor_count"] == 2
    system.close()


def test_solver_state_needs_one_body_and_the_corotated_law():
    mesh, mat = elastic_block((2, 2, 2))
    batch = tb.System([mesh, mesh], [[mat], [mat]], tb.FP64)
    with pytest.raises(capi.TalusError) as e:
        batch.use_factor(True, 32)
    assert e.value.status == capi.TL_ERR_UNSUPPORTED
    batch.close()
    system = tb.System(mesh, [mat], tb.FP64)
    system.use_factor(True, 32)
    system.set_state(tb.rest_state(mesh))
    with pytest.raises(capi.TalusError) as e:
        system.step(tb.Settings(law=tb.NEO_HOOKEAN), GRAVITY, DT)
    assert e.value.status == capi.TL_ERR_UNSUPPORTED
    system.close()


@pytest.mark.parametrize("substeps,budget", [(3, 32), (1, 0)])
def test_factored_substeps_and_budget_rules_match_oracle(substeps, budget):
    """Several substeps per step (a frame per substep, substepsSinceRefresh
    and meanIterations per substep) and a budget of 0 (the iteration cap
    itself, solver.cc:3814-3817) follow the oracle."""
    mesh, mat = plastic_block((8, 4, 4))
    settings = tb.Settings(substeps=substeps)
    errors, greps, oreps, gstats, ostats, _ = run_factored(tb.FP64, mesh, mat, settings, 3, budget=budget)
    assert max(errors) <= 1e-8, errors
    assert [r["cg_iterations"] for r in greps] == [r["cg_iterations"] for r in oreps]
    assert_same_counters(gstats, ostats)
    assert gstats["substeps_since_refresh"] == 3 * substeps
