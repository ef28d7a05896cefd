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


def run_batch_form(meshes, mats, precision, form, settings, steps):
    s = tb.System(meshes, mats, precision)
    s.set_solver(form)
    for i, m in enumerate(meshes):
        s.set_state(tb.rest_state(m), i)
    counts = []
    for _ in range(steps):
        counts.append([r.cg_iterations for r in s.step(settings, GRAVITY, DT)])
    states = [s.get_state(i).position for i in range(len(meshes))]
    s.close()
    return states, counts


@pytest.mark.parametrize("law", [tb.COROTATED, tb.NEO_HOOKEAN])
def test_pipelined_batched_pcg_equals_the_two_phase_order(law):
    """The batched PCG on the assembled matrix in the pipelined arrangement
    (one grid barrier per iteration, kPcgBatchSellPipe) and in the textbook
    order (two barriers, kPcgBatchSell) take the same iterates in exact
    arithmetic.  FP64, a ragged batch solved to 1e-4 (past the default cap of
    64): the same iteration counts and positions within 1e-10."""
    meshes, mats = tb.mesh.batch_bodies(count=7, seed=19, lo=3, hi=7)
    settings = tb.Settings(law=law, tolerance=1e-4, cg_iterations=2000)
    piped, piped_counts = run_batch_form(meshes, mats, tb.FP64, "assembled-pipelined", settings, 5)
    split, split_counts = run_batch_form(meshes, mats, tb.FP64, "assembled-two-phase", settings, 5)
    assert piped_counts == split_counts
    assert max(max(c) for c in piped_counts) > 64
    for i, m in enumerate(meshes):
        scale = np.linalg.norm(split[i] - m.rest_positions, axis=1).max()
        assert np.linalg.norm(piped[i] - split[i], axis=1).max() <= 1e-10 * scale, i


def test_pipelined_and_two_phase_orders_agree_at_a_tight_tolerance():
    """Solved to 1e-8 the two orders' residual recurrences (rounded
    differently) may cross the tolerance an iteration apart; the converged
    positions agree to the tolerance."""
    meshes, mats = tb.mesh.batch_bodies(count=7, seed=19, lo=3, hi=7)
    settings = tb.Settings(tolerance=1e-8, cg_iterations=4000)
    piped, piped_counts = run_batch_form(meshes, mats, tb.FP64, "assembled-pipelined", settings, 4)
    split, split_counts = run_batch_form(meshes, mats, tb.FP64, "assembled-two-phase", settings, 4)
    for a, b in zip(piped_counts, split_counts):
        assert max(abs(x - y) for x, y in zip(a, b)) <= 2
    for i, m in enumerate(meshes):
        scale = np.linalg.norm(split[i] - m.rest_positions, axis=1).max()
        assert np.linalg.norm(piped[i] - split[i], axis=1).max() <= 1e-7 * scale, i


def test_fp32_mixed_batch_follows_the_fp64_batch_at_a_converged_tolerance():
    """The FP32-mixed batch (two-phase order) against the FP64 batch
    (pipelined order), both solved to 1e-6 on soft bodies that move by
    millimetres or more: within 1e-5 of the displacement, no solve at the cap."""
    meshes, _ = tb.mesh.batch_bodies(count=7, seed=23, lo=3, hi=7)
    mats = [[tb.PhysicalMaterial(density=1000.0, youngs_modulus=e, poissons_ratio=0.3)]
            for e in (2e4, 5e4, 1e5, 3e4, 8e4, 4e4, 6e4)]
    settings = tb.Settings(tolerance=1e-6, cg_iterations=4000)
    ref, _ = run_batch_form(meshes, mats, tb.FP64, "assembled", settings, 5)
    got, counts = run_batch_form(meshes, mats, tb.FP32_MIXED, "assembled", settings, 5)
    assert max(max(c) for c in counts) < 4000
    for i, m in enumerate(meshes):
        scale = np.linalg.norm(ref[i] - m.rest_positions, axis=1).max()
        assert scale > 1e-3
        assert np.linalg.norm(got[i] - ref[i], axis=1).max() <= 1e-5 * scale, i


@pytest.mark.parametrize("precision", [tb.FP64, tb.FP32_MIXED])
def test_graph_replayed_batch_equals_launched_batch(precision):
    """A batched elastic step replayed from a CUDA graph (device-side substep
    choice, masked passes) gives bitwise the state of plain launches."""
    meshes, mats = tb.mesh.batch_bodies(count=6, seed=11, lo=3, hi=6)
    states = []
    for graph in (True, False):
        s = tb.System(meshes, mats, precision)
        s.tune(graph=graph)
        for i, m in enumerate(meshes):
            s.set_state(tb.rest_state(m), i)
        for _ in range(5):
            reps = s.step(tb.Settings(), GRAVITY, DT)
        assert all(r.cg_iterations > 0 for r in reps)
        states.append(np.concatenate([s.get_state(i).position.ravel() for i in range(len(meshes))]))
        s.close()
    assert np.array_equal(states[0], states[1])


def test_profiled_graph_step_reports_kernel_class_times():
    """TL_FLAG_PROFILE events inside a captured graph fire on every replay."""
    meshes, mats = tb.mesh.batch_bodies(count=4, seed=12, lo=3, hi=5)
    s = tb.System(meshes, mats, tb.FP32_MIXED)
    for i, m in enumerate(meshes):
        s.set_state(tb.rest_state(m), i)
    for _ in range(3):
        reps = s.step(tb.Settings(profile=True), GRAVITY, DT)
        r = reps[0]
        assert r.element_seconds > 0 and r.pcg_seconds > 0
        assert r.element_seconds + r.assemble_seconds + r.pcg_seconds <= r.device_seconds * 1.01
    s.close()


@pytest.mark.parametrize("blocks", [1, 2])
def test_persistent_grid_shape_does_not_change_the_single_body_result(blocks):
    """tl_system_tune caps the persistent grid; results stay within FP64 rounding."""
    mesh, mat = elastic_block()
    out = []
    for cap in (0, blocks):
        s = tb.System(mesh, [mat], tb.FP64)
        s.tune(pcg_blocks_per_sm=cap)
        s.set_state(tb.rest_state(mesh))
        for _ in range(4):
            s.step(tb.Settings(), GRAVITY, DT)
        out.append(s.get_state().position)
        s.close()
    scale = np.linalg.norm(out[0] - mesh.rest_positions, axis=1).max()
    assert np.linalg.norm(out[0] - out[1], axis=1).max() <= 1e-10 * scale


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


@pytest.mark.parametrize("form", ["elementwise", "assembled"])
def test_smallest_bodies_in_a_ragged_batch_match_the_oracle(form):
    """One-cube (6 tets, 8 nodes) and one-by-two-cube bodies between larger
    ones: node and element tiles mostly padding, one body per tile boundary.
    Each body steps as the oracle steps it alone (FP64, <= 1e-9)."""
    from oracle import pyoracle as po
    from tests.helpers import oracle_material, oracle_settings, relative_error, to_oracle

    meshes, mats = [], []
    for cells, seed in (((1, 1, 1), 21), ((5, 4, 3), 22), ((1, 2, 1), 23), ((2, 1, 1), 24)):
        m, mat = elastic_block(cells, seed=seed)
        meshes.append(m)
        mats.append([mat])
    settings = tb.Settings()
    batch = tb.System(meshes, mats, tb.FP64)
    batch.set_solver(form)
    for i, m in enumerate(meshes):
        batch.set_state(tb.rest_state(m), i)
    refs = [(to_oracle(m), po.State.rest(to_oracle(m))) for m in meshes]
    for _ in range(6):
        batch.step(settings, GRAVITY, DT)
        for (om, ost), mat in zip(refs, mats):
            po.step(po.F64, om, ost, [oracle_material(mat[0])], oracle_settings(settings), GRAVITY, DT)
    for i, (m, (_, ost)) in enumerate(zip(meshes, refs)):
        assert relative_error(batch.get_state(i).position, ost.position, m.rest_positions) <= 1e-9, i
    batch.close()


@pytest.mark.parametrize("law,damping", [(tb.COROTATED, 0.0), (tb.COROTATED, 0.02), (tb.NEO_HOOKEAN, 0.0)])
def test_host_step_treats_rotations_as_outputs(law, damping):
    """tl_step_host does not upload the committed rotations (the step writes
    each before reading it, solver.cc:1404-1547): NaN rotations in the caller's
    buffer give bitwise the same step as the rotations of the previous step,
    and come back overwritten."""
    import ctypes as C
    from talus_b200 import _capi as capi

    mesh, mat = elastic_block((6, 5, 4), seed=8)
    mat.stiffness_damping = damping
    system = tb.System(mesh, [mat], tb.FP64)
    settings = tb.Settings(law=law)
    g = np.asarray(GRAVITY, np.float64)
    results = []
    for poison in (False, True):
        st = tb.rest_state(mesh)
        arrays = {k: np.ascontiguousarray(getattr(st, k), np.float64) for k in
                  ("position", "velocity", "acceleration", "rotation", "plastic")}
        for n in range(4):
            if poison:
                arrays["rotation"][:] = np.nan
            rc = capi.lib().tl_step_host(system.handle, 0, capi.TL_DTYPE_F64,
                                         *[arrays[k].ctypes.data for k in
                                           ("position", "velocity", "acceleration", "rotation", "plastic")],
                                         C.byref(settings._c()), g.ctypes.data, DT, C.byref(capi.tl_step_report()))
            assert rc == capi.TL_OK, (poison, n, rc)
        results.append(arrays)
    system.close()
    clean, poisoned = results
    assert np.isfinite(poisoned["rotation"]).all()
    for k in clean:
        assert np.array_equal(clean[k], poisoned[k]), k


def test_host_step_moves_plastic_state_only_when_the_step_uses_it():
    """An elastic body: tl_step_host neither uploads nor downloads the plastic
    slot (the step leaves it as it is), so a NaN-filled buffer stays as passed
    and the step equals the resident one.  A yielding body's slot crosses."""
    import ctypes as C
    from talus_b200 import _capi as capi

    def host_steps(mesh, mat, poison, n=3):
        system = tb.System(mesh, [mat], tb.FP64)
        st = tb.rest_state(mesh)
        arrays = {k: np.ascontiguousarray(getattr(st, k), np.float64) for k in
                  ("position", "velocity", "acceleration", "rotation", "plastic")}
        if poison:
            arrays["plastic"][:] = np.nan
        g = np.asarray(GRAVITY, np.float64)
        for _ in range(n):
            rc = capi.lib().tl_step_host(system.handle, 0, capi.TL_DTYPE_F64,
                                         *[arrays[k].ctypes.data for k in
                                           ("position", "velocity", "acceleration", "rotation", "plastic")],
                                         C.byref(tb.Settings()._c()), g.ctypes.data, DT,
                                         C.byref(capi.tl_step_report()))
            assert rc == capi.TL_OK
        system.close()
        return arrays

    mesh, mat = elastic_block((5, 4, 4), seed=12)
    clean, poisoned = host_steps(mesh, mat, False), host_steps(mesh, mat, True)
    assert np.isnan(poisoned["plastic"]).all()
    assert np.array_equal(clean["position"], poisoned["position"])
    pmesh, pmat = plastic_block((8, 4, 4))
    moved = host_steps(pmesh, pmat, False)
    assert moved["plastic"][:, 9].max() > 0.0


@pytest.mark.parametrize("dtype", ["f32", "f64"])
def test_pinned_host_buffers_step_like_pageable_ones(dtype):
    """tl_host_register page-locks the caller's state buffers; tl_step_host
    then moves every state array by one DMA each way instead of through the
    library's staging, node arrays converted on the device.  The states are
    bitwise the same either way, for a yielding body (the plastic slot
    crosses both ways), in both caller precisions."""
    import ctypes as C
    from talus_b200 import _capi as capi

    mesh, mat = plastic_block()
    results = []
    # nothing pinned, everything pinned, and a mix (per-array choice)
    for pinned in ((), ("position", "velocity", "acceleration", "rotation", "plastic"), ("position", "plastic")):
        system = tb.System(mesh, [mat], tb.FP32_MIXED)
        st = tb.rest_state(mesh)
        np_t = np.float32 if dtype == "f32" else np.float64
        arrays = {k: np.ascontiguousarray(getattr(st, k), np_t) for k in
                  ("position", "velocity", "acceleration", "rotation", "plastic")}
        for k in pinned:
            system.context.pin(arrays[k])
        g = np.asarray(GRAVITY, np.float64)
        s_c = tb.Settings()._c()
        for _ in range(4):
            rc = capi.lib().tl_step_host(system.handle, 0,
                                         capi.TL_DTYPE_F32 if dtype == "f32" else capi.TL_DTYPE_F64,
                                         *[arrays[k].ctypes.data for k in
                                           ("position", "velocity", "acceleration", "rotation", "plastic")],
                                         C.byref(s_c), g.ctypes.data, DT, C.byref(capi.tl_step_report()))
            assert rc == capi.TL_OK
        for k in pinned:
            system.context.unpin(arrays[k])
        results.append({k: a.copy() for k, a in arrays.items()})
        system.close()
    for r in results[1:]:
        for k in results[0]:
            assert np.array_equal(results[0][k], r[k]), k
    assert (results[1]["plastic"][:, 9] > 0).any()  # the plastic slot crossed
