"""The oracle's solver state (its restatement of SystemFactor and the
factor control of deformable::step), on the CPU: the factor conditions the
same equations the block-Jacobi PCG solves, far better, and its refresh
rules and counters behave as solver.cc:3639-3655, 3808-3910 state them."""
import numpy as np

import talus_b200 as tb
from oracle import pyoracle as po
from tests.helpers import DT, GRAVITY, elastic_block, oracle_material, oracle_settings, plastic_block, relative_error, \
    to_oracle


def run(mesh, mat, settings, steps, solver=None, dt=DT):
    om = to_oracle(mesh)
    state = po.State.rest(om)
    reps = [po.step(po.F64, om, state, [oracle_material(mat)], oracle_settings(settings), GRAVITY, dt,
                    solver=solver).as_dict() for _ in range(steps)]
    return state, reps


def test_factor_solves_the_same_equations_in_fewer_iterations():
    mesh, mat = elastic_block((6, 6, 6))
    settings = tb.Settings(tolerance=1e-9, cg_iterations=500)
    plain, preps = run(mesh, mat, settings, 3)
    solver = po.Solver(32)
    fact, freps = run(mesh, mat, settings, 3, solver)
    assert relative_error(fact.position, plain.position, mesh.rest_positions) <= 1e-6
    assert sum(r["cg_iterations"] for r in freps) * 5 < sum(r["cg_iterations"] for r in preps)
    st = solver.stats()
    assert st["ready"] == 1 and st["refactor_count"] == 1 and st["generation"] == 1
    assert st["rows"] == 3 * mesh.nodes and st["substeps_since_refresh"] == 3
    assert st["factor_applications"] == sum(r["cg_iterations"] for r in freps) + sum(r["substeps"] for r in freps) * 3


def test_system_nonzeros_count_the_full_scalar_system():
    """systemNonZeros: 9 entries per coupled pair of free nodes and per free
    node, 3 per anchored node (factor.cc:441-457 setFromTriplets)."""
    mesh, mat = elastic_block((3, 2, 2))
    solver = po.Solver(32)
    run(mesh, mat, tb.Settings(), 1, solver)
    pairs = set()
    for t in mesh.tet_nodes:
        for a in t:
            for b in t:
                if not mesh.anchored[a] and not mesh.anchored[b]:
                    pairs.add((int(a), int(b)))
    expected = 9 * len(pairs) + 3 * int(mesh.anchored.sum())
    assert solver.stats()["system_nonzeros"] == expected


def test_capped_factored_solves_refresh_and_retry():
    mesh, mat = plastic_block((6, 3, 3))
    solver = po.Solver(2)
    _, reps = run(mesh, mat, tb.Settings(), 3, solver)
    st = solver.stats()
    assert st["retries"] > 0 and st["retries"] == st["refactors"] == st["refresh_requests"]
    assert st["refactor_count"] == 1 + st["retries"] and st["retry_count"] == st["retries"]
    assert st["wasted_iterations"] >= 2 * st["retries"]


def test_a_new_step_length_refreshes_the_factor():
    mesh, mat = elastic_block((3, 3, 3))
    solver = po.Solver(32)
    om = to_oracle(mesh)
    state = po.State.rest(om)
    for dt in (DT, DT, DT / 2):
        po.step(po.F64, om, state, [oracle_material(mat)], oracle_settings(tb.Settings()), GRAVITY, dt, solver=solver)
    assert solver.stats()["refactor_count"] == 2


def test_damped_factor_conditions_the_damped_system():
    """With stiffness damping the factor holds the damping blocks too
    (factor.cc:346-366): the factored step solves the same damped equations."""
    mesh, _ = elastic_block((5, 5, 5))
    mat = tb.PhysicalMaterial(density=1000.0, youngs_modulus=1e6, poissons_ratio=0.3, stiffness_damping=0.02)
    settings = tb.Settings(tolerance=1e-9, cg_iterations=500)
    plain, preps = run(mesh, mat, settings, 3)
    solver = po.Solver(32)
    fact, freps = run(mesh, mat, settings, 3, solver)
    assert relative_error(fact.position, plain.position, mesh.rest_positions) <= 1e-6
    assert sum(r["cg_iterations"] for r in freps) * 4 < sum(r["cg_iterations"] for r in preps)
    assert solver.stats()["refactor_count"] == 1


def test_factored_step_in_the_reference_arithmetic_follows_fp64():
    """The FP32 restatement (the reference's glm arithmetic) with a solver
    state stays near the FP64 step without one, at the reference's own FP32
    error level."""
    mesh, mat = plastic_block((8, 4, 4))
    om = to_oracle(mesh)
    st32, st64 = po.State.rest(om), po.State.rest(om)
    solver = po.Solver(32)
    for _ in range(3):
        po.step(po.F32, om, st32, [oracle_material(mat)], oracle_settings(tb.Settings()), GRAVITY, DT, solver=solver)
        po.step(po.F64, om, st64, [oracle_material(mat)], oracle_settings(tb.Settings()), GRAVITY, DT)
    assert relative_error(st32.position, st64.position, mesh.rest_positions) <= 1e-4
    assert solver.stats()["refactor_count"] == 1
