"""Stiffness damping on the GPU against the oracle (factor.cc:755-855,
solver.cc:625-902): the rigid fit and viscous force of the element pass, the
damped matvec of both PCG kernels and the damped preconditioner blocks.

Bars as in test_gpu_parity: FP64 GPU vs FP64 oracle <= 1e-9 (elastic) and
1e-8 (plastic Newton path); FP32-mixed vs FP64 oracle <= 1e-5.
"""
import numpy as np
import pytest

import talus_b200 as tb
from oracle import pyoracle as po
from tests.helpers import (DT, GRAVITY, elastic_block, oracle_material, oracle_settings, plastic_block,
                           relative_error, run_gpu, run_oracle, to_oracle)

pytestmark = pytest.mark.gpu


def damped(mat, tau):
    return tb.PhysicalMaterial(density=mat.density, youngs_modulus=mat.youngs_modulus,
                               poissons_ratio=mat.poissons_ratio, stiffness_damping=tau,
                               yield_stress=mat.yield_stress, hardening_modulus=mat.hardening_modulus)


@pytest.mark.parametrize("precision,tol", [(tb.FP64, 1e-9), (tb.FP32_MIXED, 1e-5)])
def test_damped_elastic_block_matches_oracle(precision, tol):
    mesh, mat = elastic_block()
    mat = damped(mat, 0.02)
    settings = tb.Settings()
    ref, got = [], []
    run_oracle(po.F64, mesh, mat, settings, 12, record=ref)
    run_gpu(precision, mesh, mat, settings, 12, record=got)
    for step, (x, r) in enumerate(zip(got, ref)):
        assert relative_error(x, r, mesh.rest_positions) <= tol, step


def test_damped_plastic_block_matches_oracle():
    mesh, mat = plastic_block()
    mat = damped(mat, 0.005)
    settings = tb.Settings()
    ref, got = [], []
    _, oreps = run_oracle(po.F64, mesh, mat, settings, 8, record=ref)
    _, greps = run_gpu(tb.FP64, mesh, mat, settings, 8, record=got)
    for step, (x, r) in enumerate(zip(got, ref)):
        assert relative_error(x, r, mesh.rest_positions) <= 1e-8, step
    assert [r["plastic_evaluations"] for r in greps] == [r["plastic_evaluations"] for r in oreps]


def test_damping_on_one_lane_only():
    mesh, mat = elastic_block((8, 6, 6), seed=4)
    mesh.material[: mesh.tets // 2] = 1  # the first half of the tets takes the damped lane
    mats = [mat, damped(mat, 0.05)]
    om = to_oracle(mesh)
    ost = po.State.rest(om)
    sys_ = tb.System(mesh, mats, tb.FP64)
    sys_.set_state(tb.rest_state(mesh))
    for _ in range(10):
        po.step(po.F64, om, ost, [oracle_material(m) for m in mats], oracle_settings(tb.Settings()), GRAVITY, DT)
        sys_.step(tb.Settings(), GRAVITY, DT)
    assert relative_error(sys_.get_state().position, ost.position, mesh.rest_positions) <= 1e-9


def test_batched_damped_bodies_match_single_systems():
    meshes, mats = tb.mesh.batch_bodies(count=5, seed=8, lo=3, hi=6)
    mats = [[damped(m[0], 0.01 * (i % 2))] for i, m in enumerate(mats)]
    batch = tb.System(meshes, mats, tb.FP64)
    singles = [tb.System(m, mt, tb.FP64) for m, mt in zip(meshes, mats)]
    for i, m in enumerate(meshes):
        batch.set_state(tb.rest_state(m), i)
        singles[i].set_state(tb.rest_state(m))
    for _ in range(6):
        batch.step(tb.Settings(), GRAVITY, DT)
        for s in singles:
            s.step(tb.Settings(), GRAVITY, DT)
    for i, (m, s) in enumerate(zip(meshes, singles)):
        ref = s.get_state().position
        assert relative_error(batch.get_state(i).position, ref, m.rest_positions) <= 1e-10, i


def test_damping_needs_the_corotated_law():
    mesh, mat = elastic_block((3, 3, 3))
    s = tb.System(mesh, [damped(mat, 0.02)], tb.FP64)
    s.set_state(tb.rest_state(mesh))
    with pytest.raises(tb._capi.TalusError) as e:
        s.step(tb.Settings(law=tb.NEO_HOOKEAN), GRAVITY, DT)
    assert e.value.status == tb._capi.TL_ERR_UNSUPPORTED
