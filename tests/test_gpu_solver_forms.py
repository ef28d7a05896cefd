"""The two forms of the single-body PCG operator (tl_system_set_solver): the
assembled 3x3 node-block matrix and the element-by-element application of
applySystem (solver.cc:904-1048).  They apply the same operator, so their
trajectories agree to rounding, and each matches the FP64 oracle at the
parity bars of test_gpu_parity."""
import numpy as np
import pytest

import talus_b200 as tb
from oracle import pyoracle as po
from tests.helpers import DT, GRAVITY, elastic_block, plastic_block, relative_error, run_oracle

pytestmark = pytest.mark.gpu


def run(form, precision, mesh, mat, settings, steps):
    s = tb.System(mesh, [mat], precision)
    s.set_solver(form)
    s.set_state(tb.rest_state(mesh))
    reports = [s.step(settings, GRAVITY, DT)[0].as_dict() for _ in range(steps)]
    x = s.get_state().position
    s.close()
    return x, reports


@pytest.mark.parametrize("law", [tb.COROTATED, tb.NEO_HOOKEAN])
def test_forms_agree_on_the_elastic_block(law):
    mesh, mat = elastic_block()
    settings = tb.Settings(law=law)
    xa, ra = run("assembled", tb.FP64, mesh, mat, settings, 10)
    xe, re = run("elementwise", tb.FP64, mesh, mat, settings, 10)
    assert relative_error(xa, xe, mesh.rest_positions) <= 1e-10
    assert [r["cg_iterations"] for r in ra] == [r["cg_iterations"] for r in re]


def test_elementwise_form_matches_the_oracle():
    mesh, mat = elastic_block()
    ref, got = [], []
    run_oracle(po.F64, mesh, mat, tb.Settings(), 8, record=ref)
    s = tb.System(mesh, [mat], tb.FP64)
    s.set_solver("elementwise")
    s.set_state(tb.rest_state(mesh))
    for _ in range(8):
        s.step(tb.Settings(), GRAVITY, DT)
        got.append(s.get_state().position)
    s.close()
    for step, (x, r) in enumerate(zip(got, ref)):
        assert relative_error(x, r, mesh.rest_positions) <= 1e-9, step


@pytest.mark.parametrize("precision,tol", [(tb.FP64, 1e-8), (tb.FP32_MIXED, 1e-5)])
def test_forms_agree_on_the_plastic_block(precision, tol):
    mesh, mat = plastic_block()
    xa, ra = run("assembled", precision, mesh, mat, tb.Settings(), 6)
    xe, re = run("elementwise", precision, mesh, mat, tb.Settings(), 6)
    assert relative_error(xa, xe, mesh.rest_positions) <= tol
    if precision == tb.FP64:
        assert [r["plastic_evaluations"] for r in ra] == [r["plastic_evaluations"] for r in re]


@pytest.mark.parametrize("precision,tol", [(tb.FP64, 1e-8), (tb.FP32_MIXED, 1e-5)])
def test_assembled_form_matches_the_oracle_on_the_plastic_block(precision, tol):
    mesh, mat = plastic_block()
    ref, got = [], []
    _, oreps = run_oracle(po.F64, mesh, mat, tb.Settings(), 6, record=ref)
    s = tb.System(mesh, [mat], precision)
    s.set_solver("assembled")
    s.set_state(tb.rest_state(mesh))
    greps = []
    for _ in range(6):
        greps.append(s.step(tb.Settings(), GRAVITY, DT)[0].as_dict())
        got.append(s.get_state().position)
    s.close()
    for step, (x, r) in enumerate(zip(got, ref)):
        assert relative_error(x, r, mesh.rest_positions) <= tol, step
    if precision == tb.FP64:
        assert [r["plastic_evaluations"] for r in greps] == [r["plastic_evaluations"] for r in oreps]


def test_forms_agree_on_a_batch():
    meshes, mats = tb.mesh.batch_bodies(count=5, seed=9, lo=3, hi=7)
    out = []
    for form in ("assembled", "elementwise"):
        s = tb.System(meshes, mats, tb.FP64)
        s.set_solver(form)
        for i, m in enumerate(meshes):
            s.set_state(tb.rest_state(m), i)
        reps = [s.step(tb.Settings(), GRAVITY, DT) for _ in range(6)]
        out.append(([s.get_state(i).position for i in range(len(meshes))],
                    [[r.cg_iterations for r in rs] for rs in reps]))
        s.close()
    for i, m in enumerate(meshes):
        assert relative_error(out[0][0][i], out[1][0][i], m.rest_positions) <= 1e-10, i
    assert out[0][1] == out[1][1]


def test_unknown_form_is_rejected():
    mesh, mat = elastic_block((3, 3, 3))
    s = tb.System(mesh, [mat], tb.FP64)
    with pytest.raises(tb._capi.TalusError) as e:
        tb._capi.check(tb._capi.lib().tl_system_set_solver(s.handle, 5), s.context.handle)
    assert e.value.status == tb._capi.TL_ERR_ARG
    s.close()


def test_pipelined_batch_order_in_fp32_mixed_follows_fp64():
    """The pipelined batched order keeps its recurrences in FP64 in both
    precisions (as the single-body kernel keeps them in registers); in
    FP32-mixed only the matrix and the published matvec input are FP32.  A
    ragged batch solved to 1e-6 stays within 1e-5 of the FP64 batch."""
    meshes, _ = tb.mesh.batch_bodies(count=6, seed=29, lo=3, hi=6)
    mats = [[tb.PhysicalMaterial(density=1000.0, youngs_modulus=e, poissons_ratio=0.3)]
            for e in (2e4, 5e4, 1e5, 3e4, 8e4, 4e4)]
    settings = tb.Settings(tolerance=1e-6, cg_iterations=4000)
    out = {}
    for precision in (tb.FP64, tb.FP32_MIXED):
        s = tb.System(meshes, mats, precision)
        s.set_solver("assembled-pipelined")
        for i, m in enumerate(meshes):
            s.set_state(tb.rest_state(m), i)
        for _ in range(4):
            reps = s.step(settings, GRAVITY, DT)
        assert all(r.cg_capped_solves == 0 for r in reps)
        out[precision] = [s.get_state(i).position for i in range(len(meshes))]
        s.close()
    for i, m in enumerate(meshes):
        ref = out[tb.FP64][i]
        scale = np.linalg.norm(ref - m.rest_positions, axis=1).max()
        assert np.linalg.norm(out[tb.FP32_MIXED][i] - ref, axis=1).max() <= 1e-5 * scale, i


def test_forms_agree_on_a_body_too_large_for_one_row_per_thread():
    """A body with more node rows than the single-body assembled PCG has
    threads (91,908 nodes) runs the assembled operator through the batched
    kernel; it agrees with the element-by-element form."""
    mesh = tb.box_mesh((68, 36, 35), voxel=0.1)
    assert mesh.nodes > 2 * 148 * 256
    mat = tb.PhysicalMaterial(density=1000.0, youngs_modulus=1e6, poissons_ratio=0.3)
    xa, ra = run("assembled", tb.FP64, mesh, mat, tb.Settings(), 3)
    xe, re = run("elementwise", tb.FP64, mesh, mat, tb.Settings(), 3)
    assert relative_error(xa, xe, mesh.rest_positions) <= 1e-10
    assert [r["cg_iterations"] for r in ra] == [r["cg_iterations"] for r in re]


@pytest.mark.parametrize("precision", [tb.FP64, tb.FP32_MIXED])
def test_launch_shapes_give_bitwise_the_same_step(precision):
    """tl_system_tune_shape changes how many column slots of a matrix row are
    requested per round trip and how many blocks per SM the batched kernels
    run; the additions are the same, so the state is bitwise the same, for a
    single body (kPcgSell) and a ragged batch (both batched orders)."""
    mesh, mat = plastic_block()
    meshes, mats = tb.mesh.batch_bodies(count=5, seed=31, lo=3, hi=6)
    forms = ["assembled-two-phase", "assembled-pipelined"]
    cases = [([mesh], [[mat]], "assembled", [(0, 0), (2, 0), (4, 0)])]
    cases += [(meshes, mats, form, [(0, 0), (4, 3), (2, 3), (4, 4)]) for form in forms]
    for ms, mt, form, shapes in cases:
        results = []
        for rg, bb in shapes:
            s = tb.System(ms, mt, precision)
            s.set_solver(form)
            s.tune_shape(rg, bb)
            for i, m in enumerate(ms):
                s.set_state(tb.rest_state(m), i)
            for _ in range(3):
                s.step(tb.Settings(), GRAVITY, DT)
            results.append(np.concatenate([s.get_state(i).position.ravel() for i in range(len(ms))]))
            s.close()
        for r in results[1:]:
            assert np.array_equal(r, results[0]), form


def test_launch_shape_values_are_checked():
    mesh, mat = elastic_block((3, 3, 3))
    s = tb.System(mesh, [mat], tb.FP64)
    for knob, value in ((tb._capi.TL_SHAPE_ROW_GROUP, 3), (tb._capi.TL_SHAPE_BATCH_BLOCKS, 5), (7, 0)):
        with pytest.raises(tb._capi.TalusError) as e:
            tb._capi.check(tb._capi.lib().tl_system_tune_shape(s.handle, knob, value), s.context.handle)
        assert e.value.status == tb._capi.TL_ERR_ARG
    s.close()
