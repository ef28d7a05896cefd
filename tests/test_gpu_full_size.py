"""The benchmark workloads at their full sizes.

* plastic block against the FP64 oracle: the oracle's first two steps of the
  393,216-tet block (17 and 33 Newton evaluations, one to two minutes per
  step on one CPU core) are stored in tests/golden/full_plastic_block.npz
  (every 8th node, sums over all nodes, the step counts).  The GPU steps the
  block with the assembled operator (kSellAssemble, kPcgSell) at the tile,
  slice and grid shapes the benchmark times: FP64 within 1e-8 relative
  displacement with the same Newton evaluation and PCG iteration counts,
  FP32-mixed within 1e-5.

The rest is checked through properties that hold at any size:

* plastic block, 64x32x32 cubes (393,216 tets, 70,785 nodes), 10 steps:
  FP32-mixed within 1e-5 relative displacement of FP64 at every step; the
  pushed and pinned faces follow their prescribed motion exactly; plastic
  strain appears and stays finite and non-negative; a second FP32-mixed run
  is bitwise identical.
* batch, 512 bodies (7,907,508 tets, cells per axis drawn from U{4..24})
  in one system, 2 steps with every PCG solve converged (relative residual
  1e-6, the iteration cap out of reach): FP32-mixed within 1e-5 of FP64 on
  every body, pinned bases at rest.
"""
import os

import numpy as np
import pytest

import talus_b200 as tb
from talus_b200 import workloads
from tests.golden import make_golden as mg
from tests.helpers import DT, GRAVITY, relative_error

pytestmark = pytest.mark.gpu


def run(meshes, mats, precision, settings, steps, record=False):
    system = tb.System(meshes, mats, precision)
    for i, m in enumerate(meshes):
        system.set_state(tb.rest_state(m), i)
    history = []
    for _ in range(steps):
        system.step(settings, GRAVITY, DT)
        if record:
            history.append(system.get_state(0).position)
    states = [system.get_state(i) for i in range(len(meshes))]
    system.close()
    return states, history


@pytest.mark.parametrize("precision", [tb.FP64, tb.FP32_MIXED], ids=["fp64", "mixed"])
def test_plastic_block_at_full_size_matches_the_oracle(precision):
    g = np.load(os.path.join(os.path.dirname(mg.__file__), "full_plastic_block.npz"))
    mesh, mat, settings, steps = mg.full_block_case()
    np.testing.assert_allclose(mg.mesh_checksum(mesh), g["mesh_checksum"], rtol=1e-12)
    system = tb.System(mesh, [mat], precision)
    system.set_solver("assembled")
    system.set_state(tb.rest_state(mesh))
    sample = int(g["sample"])
    for k in range(steps):
        rep = system.step(settings, GRAVITY, DT)[0]
        x = system.get_state().position
        want = g["positions"][k]
        scale = g["sums"][k][3]  # max |x - X| over all nodes
        err = np.linalg.norm(x[::sample] - want, axis=1).max() / scale
        if precision == tb.FP64:
            assert err <= 1e-8, (k, err)
            np.testing.assert_allclose(mg.position_sums(x, mesh.rest_positions), g["sums"][k], rtol=1e-7)
            assert rep.plastic_evaluations == g["plastic_evaluations"][k], k
            assert rep.plastic_solves == g["plastic_solves"][k], k
            assert rep.cg_iterations == g["cg_iterations"][k], k
        else:
            assert err <= 1e-5, (k, err)
    state = system.get_state()
    system.close()
    if precision == tb.FP64:
        assert int((state.plastic[:, 9] > 0).sum()) == int(g["yielded"])
        assert state.plastic[:, 9].sum() == pytest.approx(float(g["equivalent_sum"]), rel=1e-8)


def test_plastic_block_at_full_size():
    spec = workloads.WORKLOADS["plastic-block"]
    mesh, mat = workloads.make_mesh(spec)
    assert (mesh.tets, mesh.nodes) == (393216, 70785)
    settings = tb.Settings()
    steps = 10
    (s64,), h64 = run([mesh], [[mat]], tb.FP64, settings, steps, record=True)
    (s32,), h32 = run([mesh], [[mat]], tb.FP32_MIXED, settings, steps, record=True)
    for n, (a, b) in enumerate(zip(h32, h64)):
        assert relative_error(a, b, mesh.rest_positions) <= 1e-5, n
    held = mesh.anchored != 0
    expected = mesh.rest_positions[held] + steps * DT * mesh.prescribed_velocity[held]
    np.testing.assert_allclose(s64.position[held], expected, rtol=0, atol=1e-12)
    np.testing.assert_allclose(s32.position[held], expected, rtol=0, atol=1e-6)
    eq = s64.plastic[:, 9]
    assert np.isfinite(s64.plastic).all() and eq.min() >= 0.0 and eq.max() > 0.0
    (again,), _ = run([mesh], [[mat]], tb.FP32_MIXED, settings, steps)
    assert np.array_equal(again.position, s32.position) and np.array_equal(again.plastic, s32.plastic)


def test_batch_at_full_size_converged():
    spec = workloads.WORKLOADS["batch"]
    meshes, mats = workloads.make_bodies(spec)
    assert len(meshes) == 512 and sum(m.tets for m in meshes) == 7_907_508
    settings = tb.Settings(cg_iterations=3000, tolerance=1e-6)
    s64, _ = run(meshes, mats, tb.FP64, settings, 2)
    s32, _ = run(meshes, mats, tb.FP32_MIXED, settings, 2)
    worst = max(relative_error(a.position, b.position, m.rest_positions) for a, b, m in zip(s32, s64, meshes))
    assert worst <= 1e-5, worst
    for st, m in zip(s64, meshes):
        held = m.anchored != 0
        assert np.array_equal(st.position[held], m.rest_positions[held])
