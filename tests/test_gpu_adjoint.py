"""The hand-written adjoint of the rollout (tl_rollout_adjoint).

* Gradients with respect to per-element E and initial velocity agree with
  FP64 central finite differences (h = 1e-6 relative) of the same GPU forward,
  along random directions and for single elements, through the
  torch.autograd.Function of the gradient-check harness.
* The checkpoint interval changes nothing: recomputation is bit-exact.
* A rollout with the reference's 3 reads is exactly tl_step repeated.
* The gradient against the oracle: FP64 central differences of the CPU
  restatement of the step on a small block (the reference itself has no
  gradient, so this pin is the oracle's forward, parity unpinned beyond it).
"""
import numpy as np
import pytest

import talus_b200 as tb
from talus_b200 import gradcheck
from tests.helpers import DT, GRAVITY

pytestmark = pytest.mark.gpu

FD_TOLERANCE = 1e-5  # relative, adjoint vs FP64 central differences of the converged forward


@pytest.fixture(scope="module")
def small():
    return gradcheck.make_problem(cells=5, steps=8, checkpoint_every=3)


def test_adjoint_matches_central_differences(small):
    rep = gradcheck.check(small, directions=2, elements=2)
    for c in rep["checks"]:
        assert c["rel"] <= FD_TOLERANCE, c
    assert rep["loss"] > 0


def test_checkpoint_interval_does_not_change_gradients(small):
    ref = small.gradients(small.youngs, small.v0)[1]
    for every in (1, 8):
        p = gradcheck.make_problem(cells=5, steps=8, checkpoint_every=every)
        g = p.gradients(p.youngs, p.v0)[1]
        assert np.array_equal(g.youngs, ref.youngs) and np.array_equal(g.velocity, ref.velocity), every


def test_three_read_rollout_is_repeated_steps():
    mesh = tb.box_mesh((4, 3, 5), voxel=0.1, jitter=0.01, seed=4)
    mat = tb.PhysicalMaterial(density=1000.0, youngs_modulus=2e6, poissons_ratio=0.35)
    settings = tb.Settings(law=tb.NEO_HOOKEAN)
    a = tb.System(mesh, [mat], tb.FP64)
    a.set_state(tb.rest_state(mesh))
    roll = tb.Rollout(a, steps=6, checkpoint_every=4, newton_reads=3, settings=settings, gravity=GRAVITY,
                      delta_time=DT)
    roll.forward()
    b = tb.System(mesh, [mat], tb.FP64)
    b.set_state(tb.rest_state(mesh))
    for _ in range(6):
        b.step(settings, GRAVITY, DT)
    assert np.array_equal(a.get_state().position, b.get_state().position)
    roll.close()


def test_gradient_is_pinned_by_oracle_differences():
    from oracle import pyoracle as po
    from tests.helpers import oracle_material, to_oracle

    p = gradcheck.make_problem(cells=3, steps=4, checkpoint_every=2, newton_reads=3, tolerance=1e-12)
    rng = np.random.default_rng(5)
    r = rng.standard_normal(p.mesh.tets)
    loss, g = p.gradients(p.youngs, p.v0)
    adjoint = float(np.sum(g.youngs * p.youngs * r))
    om = to_oracle(p.mesh)
    mat = oracle_material(tb.PhysicalMaterial(density=1000.0, youngs_modulus=1.0e6, poissons_ratio=0.3))
    settings = po.Settings(law=po.LAW_SNH, tolerance=1e-12, cg_iterations=4000)

    def oracle_loss(t):
        om.element_youngs = p.youngs * (1.0 + t * r)
        state = po.State.rest(om)
        for _ in range(4):
            po.step(po.F64, om, state, [mat], settings, GRAVITY, DT)
        d = state.position - p.target
        return float(np.sum(d * d))

    fd = (oracle_loss(1e-6) - oracle_loss(-1e-6)) / 2e-6
    assert abs(adjoint - fd) <= 1e-5 * abs(fd), (adjoint, fd)


def test_mixed_precision_gradient_tracks_fp64(small):
    mixed = gradcheck.make_problem(cells=5, steps=8, checkpoint_every=3, precision=tb.FP32_MIXED, tolerance=1e-6)
    ref = small.gradients(small.youngs, small.v0)[1]
    g = mixed.gradients(mixed.youngs, mixed.v0)[1]
    err = np.linalg.norm(g.youngs - ref.youngs) / np.linalg.norm(ref.youngs)
    assert err <= 1e-2, err


def test_rollout_refusals():
    mesh = tb.box_mesh((2, 2, 2), voxel=0.1)
    mat = tb.PhysicalMaterial(density=1000.0, youngs_modulus=1e6, poissons_ratio=0.3)
    s = tb.System(mesh, [mat], tb.FP64)
    with pytest.raises(tb._capi.TalusError) as e:
        tb.Rollout(s, steps=3, settings=tb.Settings(law=tb.COROTATED))
    assert e.value.status == tb._capi.TL_ERR_UNSUPPORTED
    two = tb.System([mesh, mesh], [[mat], [mat]], tb.FP64)
    with pytest.raises(tb._capi.TalusError) as e:
        tb.Rollout(two, steps=3)
    assert e.value.status == tb._capi.TL_ERR_UNSUPPORTED
    roll = tb.Rollout(s, steps=3)
    with pytest.raises(tb._capi.TalusError) as e:
        roll.adjoint(np.zeros((mesh.nodes, 3)))
    assert e.value.status == tb._capi.TL_ERR_ARG
