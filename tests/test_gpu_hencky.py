"""Finite-strain (Hencky) plasticity on the GPU (tl_system_set_plasticity)
against the oracle's restatement of plasticflow.cc:96-150, 184-247 and
263-300.

Bars as in test_gpu_parity: FP64 <= 1e-9 relative displacement and the
plastic maps and hardening variables within 1e-9, with the same count of
flowed tets every step; FP32-mixed <= 1e-5.  Both solver forms.  A batch
steps like its bodies alone; an elastic material steps as in the default
mode; the mode resets the plastic maps; the state slot round-trips.
"""
import numpy as np
import pytest

import talus_b200 as tb
from talus_b200 import _capi as capi
from oracle import pyoracle as po
from tests.helpers import DT, GRAVITY, elastic_block, oracle_material, plastic_block, relative_error, to_oracle

pytestmark = pytest.mark.gpu


def oracle_run(mesh, mat, steps):
    om = to_oracle(mesh)
    st = po.State.rest(om, hencky=True)
    settings = po.Settings(plasticity=po.PLASTICITY_HENCKY)
    record, flowed = [], []
    for _ in range(steps):
        rep = po.step(po.F64, om, st, [oracle_material(mat)], settings, GRAVITY, DT)
        record.append(st.position.copy())
        flowed.append(rep.as_dict()["yielding"])
    return st, record, flowed


def gpu_system(meshes, mats, precision, form="auto"):
    s = tb.System(meshes, mats, precision)
    s.set_solver(form)
    s.set_plasticity("hencky")
    for i, m in enumerate(s.meshes):
        s.set_state(tb.rest_state(m, hencky=True), i)
    return s


@pytest.mark.parametrize("form", ["elementwise", "assembled"])
@pytest.mark.parametrize("precision", [tb.FP64, tb.FP32_MIXED], ids=["fp64", "mixed"])
def test_hencky_block_matches_the_oracle(precision, form):
    mesh, mat = plastic_block()
    steps = 8
    ost, ref, oflowed = oracle_run(mesh, mat, steps)
    s = gpu_system([mesh], [[mat]], precision, form)
    tol = 1e-9 if precision == tb.FP64 else 1e-5
    for n in range(steps):
        rep = s.step(tb.Settings(), GRAVITY, DT)[0]
        x = s.get_state().position
        assert relative_error(x, ref[n], mesh.rest_positions) <= tol, n
        if precision == tb.FP64:
            assert rep.yielding == oflowed[n], n
            assert rep.plastic_evaluations == 0
    got = s.get_state()
    s.close()
    if precision == tb.FP64:
        assert np.abs(got.plastic[:, :9] - ost.plastic[:, :9]).max() <= 1e-9
        assert np.abs(got.plastic[:, 9] - ost.plastic[:, 9]).max() <= 1e-9 * max(1.0, ost.plastic[:, 9].max())
    else:
        assert np.abs(got.plastic[:, :9] - ost.plastic[:, :9]).max() <= 1e-4


def test_hencky_batch_steps_like_its_bodies_alone():
    a, ma = plastic_block((8, 4, 4), seed=3)
    b, mb = plastic_block((6, 5, 4), seed=4, speed=0.3)
    batch = gpu_system([a, b], [[ma], [mb]], tb.FP64)
    singles = [gpu_system([m], [[mat]], tb.FP64) for m, mat in ((a, ma), (b, mb))]
    for _ in range(5):
        reps = batch.step(tb.Settings(), GRAVITY, DT)
        for i, s in enumerate(singles):
            assert s.step(tb.Settings(), GRAVITY, DT)[0].yielding == reps[i].yielding
    for i, (m, s) in enumerate(zip((a, b), singles)):
        x, y = batch.get_state(i), s.get_state()
        assert relative_error(x.position, y.position, m.rest_positions) <= 1e-10
        assert np.abs(x.plastic - y.plastic).max() <= 1e-10
        s.close()
    batch.close()


def test_elastic_material_in_hencky_mode_is_the_default_step():
    mesh, mat = elastic_block((6, 5, 4), seed=9)
    s = gpu_system([mesh], [[mat]], tb.FP64)
    d = tb.System(mesh, [mat], tb.FP64)
    d.set_state(tb.rest_state(mesh))
    for _ in range(6):
        s.step(tb.Settings(), GRAVITY, DT)
        d.step(tb.Settings(), GRAVITY, DT)
    x, y = s.get_state(), d.get_state()
    assert relative_error(x.position, y.position, mesh.rest_positions) <= 1e-12
    assert np.array_equal(x.plastic[:, [0, 4, 8]], np.ones((mesh.tets, 3)))
    s.close()
    d.close()


def test_mode_resets_the_plastic_maps_and_the_slot_round_trips():
    mesh, mat = plastic_block((4, 3, 2))
    s = gpu_system([mesh], [[mat]], tb.FP64)
    st = tb.rest_state(mesh, hencky=True)
    rng = np.random.default_rng(5)
    st.plastic[:, :9] = (np.eye(3) + 0.01 * rng.standard_normal((mesh.tets, 3, 3))).reshape(-1, 9)
    st.plastic[:, 9] = rng.random(mesh.tets)
    s.set_state(st)
    assert np.array_equal(s.get_state().plastic, st.plastic)
    s.set_plasticity("hencky")
    reset = s.get_state().plastic
    assert np.array_equal(reset[:, :9], np.tile(np.eye(3).ravel(), (mesh.tets, 1))) and not reset[:, 9].any()
    s.close()


def test_hencky_refusals():
    mesh, mat = plastic_block((4, 3, 2))
    s = gpu_system([mesh], [[mat]], tb.FP64)
    with pytest.raises(capi.TalusError) as err:
        s.step(tb.Settings(law=tb.NEO_HOOKEAN), GRAVITY, DT)
    assert err.value.status == capi.TL_ERR_UNSUPPORTED
    assert capi.lib().tl_system_set_plasticity(s.handle, 2) == capi.TL_ERR_ARG
    s.close()
    mat.stiffness_damping = 0.01
    d = gpu_system([mesh], [[mat]], tb.FP64)
    with pytest.raises(capi.TalusError) as err:
        d.step(tb.Settings(), GRAVITY, DT)
    assert err.value.status == capi.TL_ERR_UNSUPPORTED
    d.close()


@pytest.mark.parametrize("limits", [dict(plastic_max=0.02), dict(crush_stress=2.0e4, crush_limit=0.95)],
                         ids=["cap", "crush"])
def test_flow_limits_match_the_oracle_and_hold(limits):
    """A plastic cap (plasticMax) and a crushable lane (crushStress,
    crushLimit) set through tl_system_set_flow_limits: FP64 parity with the
    oracle, and the limits hold on every tet (plasticflow.cc:196-240)."""
    mesh, mat = plastic_block()
    for k, v in limits.items():
        setattr(mat, k, v)
    steps = 8
    ost, ref, oflowed = oracle_run(mesh, mat, steps)
    s = gpu_system([mesh], [[mat]], tb.FP64)
    for n in range(steps):
        rep = s.step(tb.Settings(), GRAVITY, DT)[0]
        assert relative_error(s.get_state().position, ref[n], mesh.rest_positions) <= 1e-9, n
        assert rep.yielding == oflowed[n], n
    got = s.get_state()
    s.close()
    assert np.abs(got.plastic - ost.plastic).max() <= 1e-9 * max(1.0, np.abs(ost.plastic).max())
    stretch = np.linalg.inv(got.plastic[:, :9].reshape(-1, 3, 3))
    if "plastic_max" in limits:
        distance = np.linalg.norm(stretch - np.eye(3), axis=(1, 2))
        assert distance.max() <= limits["plastic_max"] + 1e-9 and distance.max() > 0.5 * limits["plastic_max"]
    else:
        kept = np.linalg.det(stretch)
        assert kept.min() >= limits["crush_limit"] - 1e-9 and kept.min() < 0.999


def test_flow_limit_arguments_are_checked():
    mesh, mat = plastic_block((4, 3, 2))
    s = gpu_system([mesh], [[mat]], tb.FP64)
    lib = capi.lib()
    assert lib.tl_system_set_flow_limits(s.handle, 0, 0, 1e3, 0.5, 1.0) == capi.TL_OK
    assert lib.tl_system_set_flow_limits(s.handle, 0, 1, 1e3, 0.5, 1.0) == capi.TL_ERR_ARG  # one lane only
    assert lib.tl_system_set_flow_limits(s.handle, 1, 0, 1e3, 0.5, 1.0) == capi.TL_ERR_ARG  # one body only
    assert lib.tl_system_set_flow_limits(s.handle, 0, 0, -1.0, 0.5, 1.0) == capi.TL_ERR_ARG
    assert lib.tl_system_set_flow_limits(s.handle, 0, 0, 1e3, 1.5, 1.0) == capi.TL_ERR_ARG
    assert lib.tl_system_set_flow_limits(s.handle, 0, 0, 1e3, 0.5, float("nan")) == capi.TL_ERR_ARG
    s.close()
