"""The finite-strain (Hencky) plastic flow in the oracle, CPU.

Known answers restated from the reference's own tests of returnMap and
flowLattice (tests/dynamics_strainstep_tests.cc:3090-3191), at one point: a
point inside its yield surface stays elastic; a point past it returns onto
the surface and keeps its volume, with strain = (q - yield) / (3 mu); after a
flow the elastic map's von Mises stress equals the hardened yield stress
yield + H * hardening; repeated pulls keep the plastic stretch within its cap;
repeated squeezes crush no further than the crush limit.  Then the flow
inside the oracle's tet step
(plasticflow.cc:184-247 once per step, elastic steps from the plastic rest
shape of plasticflow.cc:263-300).
"""
import numpy as np
import pytest

import talus_b200 as tb
from oracle import pyoracle as po
from tests.helpers import DT, GRAVITY, elastic_block, oracle_material, plastic_block, relative_error, to_oracle


def moduli(youngs, poisson):
    """(shear, bulk) of the tet law (lame, material.cc:71-78)."""
    nu = min(max(poisson, 0.0), 0.49)
    lam = youngs * nu / ((1 + nu) * (1 - 2 * nu))
    mu = youngs / (2 * (1 + nu))
    return mu, lam + 2 * mu / 3


def columns(*cols):
    """A matrix from its columns (glm::dmat3's constructor order)."""
    return np.array(cols, np.float64).T


def test_point_inside_yield_surface_stays_elastic():
    # dynamics_strainstep_tests.cc:3090-3094
    elastic = columns((1.0, 0.0, 0.0), (0.001, 1.0, 0.0), (0.0, 0.0, 1.0))
    assert po.hencky_return(elastic, 1.0e5, 1.0e3) is None


def test_point_past_yield_returns_onto_the_surface_and_keeps_its_volume():
    # dynamics_strainstep_tests.cc:3096-3105
    elastic = columns((1.05, 0.02, 0.0), (0.2, 0.98, 0.01), (0.0, 0.03, 1.01))
    mapped = po.hencky_return(elastic, 1.0e5, 2.0e3)
    assert mapped is not None
    back, strain, trial = mapped
    assert abs(po.hencky_von_mises(back, 1.0e5) - 2.0e3) <= 1.0e-9 * 2.0e3
    assert abs(np.linalg.det(back) - np.linalg.det(elastic)) <= 1.0e-12
    assert abs(strain - (trial - 2.0e3) / 3.0e5) <= 1.0e-12


@pytest.mark.parametrize("hardening", [0.0, 5.0e4])
def test_flow_hardens_as_the_hardening_modulus_says(hardening):
    # dynamics_strainstep_tests.cc:3107-3135 at one point: a shear x += 0.2 y
    shear, yield_stress = 1.0e5, 2.0e3
    mat = po.material(youngs=2.7e5, poisson=0.35, yield_stress=yield_stress, hardening=hardening)
    deformation = np.eye(3)
    deformation[0, 1] = 0.2
    changed, plastic, alpha = po.hencky_flow(deformation, np.eye(3), 0.0, shear, 3e5, mat)
    assert changed and alpha > 0.0
    yield_now = yield_stress + hardening * alpha
    assert abs(po.hencky_von_mises(deformation @ plastic, shear) - yield_now) <= 1.0e-6 * yield_now
    # the return is deviatoric: the plastic map keeps volume
    assert abs(np.linalg.det(plastic) - 1.0) <= 1e-12
    # flowing again from the returned state moves nothing
    again, plastic2, alpha2 = po.hencky_flow(deformation, plastic, alpha, shear, 3e5, mat)
    assert not again and np.array_equal(plastic2, plastic) and alpha2 == alpha


def test_inverted_or_elastic_points_do_not_flow():
    mat = po.material(youngs=2.7e5, poisson=0.35, yield_stress=1e3)
    flipped = np.diag([1.0, 1.0, -0.5])
    assert not po.hencky_flow(flipped, np.eye(3), 0.0, 1e5, 3e5, mat)[0]
    small = np.eye(3)
    small[0, 1] = 1e-4
    assert not po.hencky_flow(small, np.eye(3), 0.0, 1e5, 3e5, mat)[0]


def test_plastic_stretch_stays_within_its_cap():
    # dynamics_strainstep_tests.cc:3137-3167: clay(5e3, 50) (nu 0.35, plasticMax 1)
    # pulled to stretch 2..7 along x, 1/stretch along y, one flow per pull
    mat = po.material(youngs=5.0e3, poisson=0.35, yield_stress=50.0, plastic_max=1.0)
    shear, bulk = moduli(5.0e3, 0.35)
    plastic, alpha = np.eye(3), 0.0
    for pull in range(1, 7):
        stretch = 1.0 + pull
        _, plastic, alpha = po.hencky_flow(np.diag([stretch, 1.0 / stretch, 1.0]), plastic, alpha, shear, bulk, mat)
    distance = np.linalg.norm(np.linalg.inv(plastic) - np.eye(3))
    assert distance > 0.5 and distance <= 1.0 + 1e-9


def test_squeezed_point_crushes_no_further_than_its_limit():
    # dynamics_strainstep_tests.cc:3169-3191: clay(1e5, 1e9), crushStress 1e3,
    # crushLimit 0.7, squeezed to 0.6 of its size ten times
    mat = po.material(youngs=1.0e5, poisson=0.35, yield_stress=1.0e9, crush_stress=1.0e3, crush_limit=0.7)
    shear, bulk = moduli(1.0e5, 0.35)
    plastic, alpha = np.eye(3), 0.0
    for _ in range(10):
        _, plastic, alpha = po.hencky_flow(0.6 * np.eye(3), plastic, alpha, shear, bulk, mat)
    kept = np.linalg.det(np.linalg.inv(plastic))
    assert kept < 0.99 and kept >= 0.7 - 1e-9
    assert alpha == 0.0  # compaction alone: nothing returned, no hardening


def run(mesh, mat, plasticity, steps, law=po.LAW_COROTATED):
    om = to_oracle(mesh)
    st = po.State.rest(om, hencky=plasticity == po.PLASTICITY_HENCKY)
    settings = po.Settings(law=law, plasticity=plasticity)
    reports = [po.step(po.F64, om, st, [oracle_material(mat)], settings, GRAVITY, DT).as_dict() for _ in range(steps)]
    return st, reports


def test_hencky_block_flows_isochorically_and_hardens():
    mesh, mat = plastic_block()
    st, reports = run(mesh, mat, po.PLASTICITY_HENCKY, 6)
    P = st.plastic[:, :9].reshape(-1, 3, 3)
    assert all(r["yielding"] > 0 for r in reports)
    assert all(r["plastic_evaluations"] == 0 for r in reports)  # elastic steps: no Newton loop
    assert np.abs(np.linalg.det(P) - 1.0).max() <= 1e-12
    assert st.plastic[:, 9].min() >= 0.0 and st.plastic[:, 9].max() > 0.0
    held = mesh.anchored != 0
    np.testing.assert_allclose(st.position[held], mesh.rest_positions[held] + 6 * DT * mesh.prescribed_velocity[held],
                               rtol=0, atol=1e-12)


def test_hencky_mode_without_yield_is_the_elastic_step():
    """From P = I the plastic rest is the authored rest: an elastic material
    steps as in the small-strain mode (the corotated offsets come from the
    rest corners rebuilt from Dm^-1, so they agree to rounding)."""
    mesh, mat = elastic_block((6, 5, 4), seed=9)
    a, _ = run(mesh, mat, po.PLASTICITY_HENCKY, 8)
    b, _ = run(mesh, mat, po.PLASTICITY_SMALL_STRAIN, 8)
    assert relative_error(a.position, b.position, mesh.rest_positions) <= 1e-12
    assert np.array_equal(a.plastic[:, [0, 4, 8]], np.ones((mesh.tets, 3)))


def test_hencky_is_refused_with_the_snh_law_and_with_damping():
    mesh, mat = plastic_block((4, 2, 2))
    with pytest.raises(RuntimeError):
        run(mesh, mat, po.PLASTICITY_HENCKY, 1, law=po.LAW_SNH)
    mat.stiffness_damping = 0.01
    with pytest.raises(RuntimeError):
        run(mesh, mat, po.PLASTICITY_HENCKY, 1)


@pytest.mark.parametrize("limits", [dict(plastic_max=0.02), dict(crush_stress=2.0e4, crush_limit=0.95)],
                         ids=["cap", "crush"])
def test_flow_limits_hold_through_a_block_step(limits):
    """In the oracle's step, the cap and the crush limit hold on every tet of a
    pushed block, and a limit that binds changes the trajectory."""
    mesh, mat = plastic_block()
    free, _ = run(mesh, mat, po.PLASTICITY_HENCKY, 6)
    for k, v in limits.items():
        setattr(mat, k, v)
    st, reports = run(mesh, mat, po.PLASTICITY_HENCKY, 6)
    stretch = np.linalg.inv(st.plastic[:, :9].reshape(-1, 3, 3))
    if "plastic_max" in limits:
        assert np.linalg.norm(stretch - np.eye(3), axis=(1, 2)).max() <= limits["plastic_max"] + 1e-9
        assert np.linalg.norm(np.linalg.inv(free.plastic[:, :9].reshape(-1, 3, 3)) - np.eye(3),
                              axis=(1, 2)).max() > limits["plastic_max"]
    else:
        assert np.linalg.det(stretch).min() >= limits["crush_limit"] - 1e-9
        assert np.linalg.det(stretch).min() < 0.999
    assert relative_error(st.position, free.position, mesh.rest_positions) > 1e-6
