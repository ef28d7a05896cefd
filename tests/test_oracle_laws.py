"""Known-answer tests that pin the oracle (CPU, no GPU).

The reference has no test of its tet path (nothing calls deformable::step),
so these restate, for one tet, the law tests the reference does have:
tests/neohookean_tests.cc:115-199 (rest / rigid motion / small strain /
inversion of the neo-Hookean law), tests/dynamics_tests.cc:119-336 (FP64 vs
FP32 agreement, Hessian vs finite differences, zero force under rigid
motion, finite terms when inverted), tests/dynamics_strainstep_tests.cc:
3090-3104 (a point inside the yield surface stays elastic; a point past it
returns onto the surface) plus the closed forms of linear elasticity and of
the generalized-alpha recurrence for free fall.
"""
import math

import numpy as np
import pytest

from oracle import pyoracle as po

RUBBER = po.material(1000.0, 1e6, 0.4)
REST = np.array([[0.0, 0.0, 0.0], [0.1, 0.0, 0.0], [0.0, 0.1, 0.0], [0.0, 0.0, 0.1]])


def rest_inverse(rest=REST):
    return np.linalg.inv(np.stack([rest[1] - rest[0], rest[2] - rest[0], rest[3] - rest[0]], axis=1))


def volume(rest=REST):
    return np.linalg.det(np.stack([rest[1] - rest[0], rest[2] - rest[0], rest[3] - rest[0]], axis=1)) / 6.0


def rotation(angle, axis):
    axis = np.asarray(axis, float) / np.linalg.norm(axis)
    k = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    return np.eye(3) + math.sin(angle) * k + (1 - math.cos(angle)) * k @ k


def mapped(F, shift=(0.0, 0.0, 0.0)):
    return REST @ F.T + np.asarray(shift)


def lame(m):
    nu = min(max(m.poissons_ratio, 0.0), 0.49)
    return m.youngs_modulus * nu / ((1 + nu) * (1 - 2 * nu)), m.youngs_modulus / (2 * (1 + nu))


SCALE = lame(RUBBER)[1] * 0.1 * 0.1  # mu * edge^2: force unit


@pytest.mark.parametrize("precision,tol", [(po.F64, 1e-9), (po.F32, 1e-5)])
def test_snh_tet_carries_no_force_at_rest_or_rigidly_moved(precision, tol):
    out = po.snh_tet(precision, REST, REST, rest_inverse(), volume(), RUBBER)
    assert np.abs(out["force"]).max() < tol * SCALE
    assert abs(out["energy"]) < tol * SCALE * 0.1
    turned = mapped(rotation(0.7, (1, 2, 3)), (0.3, -0.1, 0.2))
    out = po.snh_tet(precision, turned, REST, rest_inverse(), volume(), RUBBER)
    assert np.abs(out["force"]).max() < 10 * tol * SCALE


def test_snh_tet_matches_corotated_at_small_strain():
    strain = np.array([[2.0e-4, 0.7e-4, -0.4e-4], [0.7e-4, -1.1e-4, 0.9e-4], [-0.4e-4, 0.9e-4, 0.6e-4]])
    deformed = mapped(np.eye(3) + strain)
    neo = po.snh_tet(po.F64, deformed, REST, rest_inverse(), volume(), RUBBER)
    cor = po.tet_trial(po.F64, deformed, REST, rest_inverse(), volume(), RUBBER, po.ROTATION_POLAR)
    scale = np.abs(cor["force"]).max()
    assert scale > 0
    assert np.linalg.norm(neo["force"] - cor["force"], axis=1).max() < 2e-3 * scale
    assert abs(neo["energy"] - cor["energy"]) < 2e-3 * cor["energy"]


def test_inverted_snh_tet_keeps_finite_forces():
    mirror = np.diag([-1.0, 1.0, 1.0])
    out = po.snh_tet(po.F64, mapped(mirror), REST, rest_inverse(), volume(), RUBBER)
    assert np.all(np.isfinite(out["force"]))
    assert math.isfinite(out["energy"]) and out["energy"] > 0
    assert np.abs(out["force"]).max() > 0


def test_snh_fp64_and_fp32_agree():
    F = np.array([[1.05, 0.02, 0.0], [0.2, 0.98, 0.01], [0.0, 0.03, 1.01]])
    a = po.snh_tet(po.F64, mapped(F), REST, rest_inverse(), volume(), RUBBER)
    b = po.snh_tet(po.F32, mapped(F), REST, rest_inverse(), volume(), RUBBER)
    largest = np.abs(a["force"]).max()
    assert np.abs(a["force"] - b["force"]).max() <= 1e-4 * largest
    assert abs(a["energy"] - b["energy"]) <= 1e-4 * abs(a["energy"])


def test_snh_tangent_matches_finite_differences_of_the_force():
    F = np.array([[1.05, 0.02, 0.0], [0.2, 0.98, 0.01], [0.0, 0.03, 1.01]])
    x = mapped(F)
    out = po.snh_tet(po.F64, x, REST, rest_inverse(), volume(), RUBBER)
    K = out["hessian"]
    scale = np.abs(K).max()
    h = 1e-7
    for col in range(12):
        plus, minus = x.copy().ravel(), x.copy().ravel()
        plus[col] += h
        minus[col] -= h
        fp = po.snh_tet(po.F64, plus.reshape(4, 3), REST, rest_inverse(), volume(), RUBBER)["force"].ravel()
        fm = po.snh_tet(po.F64, minus.reshape(4, 3), REST, rest_inverse(), volume(), RUBBER)["force"].ravel()
        fd = -(fp - fm) / (2 * h)  # K = -d force / d x
        assert np.abs(fd - K[:, col]).max() <= 1e-6 * scale


def test_snh_energy_gradient_is_minus_the_force():
    F = np.array([[1.1, 0.05, 0.0], [0.0, 0.95, 0.02], [0.01, 0.0, 1.03]])
    x = mapped(F)
    force = po.snh_tet(po.F64, x, REST, rest_inverse(), volume(), RUBBER)["force"].ravel()
    h = 1e-7
    for col in range(12):
        plus, minus = x.copy().ravel(), x.copy().ravel()
        plus[col] += h
        minus[col] -= h
        ep = po.snh_tet(po.F64, plus.reshape(4, 3), REST, rest_inverse(), volume(), RUBBER)["energy"]
        em = po.snh_tet(po.F64, minus.reshape(4, 3), REST, rest_inverse(), volume(), RUBBER)["energy"]
        assert abs(-(ep - em) / (2 * h) - force[col]) <= 1e-6 * np.abs(force).max()


@pytest.mark.parametrize("precision,tol", [(po.F64, 1e-9), (po.F32, 2e-4)])
def test_corotated_tet_rigid_motion_has_no_force(precision, tol):
    turned = mapped(rotation(1.1, (0.3, -1, 0.4)), (1.0, 2.0, -0.5))
    out = po.tet_trial(precision, turned, REST, rest_inverse(), volume(), RUBBER, po.ROTATION_POLAR)
    assert np.abs(out["force"]).max() < tol * SCALE
    R = rotation(1.1, (0.3, -1, 0.4))
    assert np.abs(out["rotation"] - R).max() < (1e-9 if precision == po.F64 else 1e-5)


def test_corotated_tet_is_linear_elasticity_at_small_strain():
    eps = np.array([[1e-6, 2e-7, 0], [2e-7, -3e-7, 1e-7], [0, 1e-7, 5e-7]])
    out = po.tet_trial(po.F64, mapped(np.eye(3) + eps), REST, rest_inverse(), volume(), RUBBER, po.ROTATION_POLAR)
    lam, mu = lame(RUBBER)
    sigma = lam * np.trace(eps) * np.eye(3) + 2 * mu * eps
    g = np.vstack([-rest_inverse().sum(axis=0), rest_inverse()])
    expected = -volume() * g @ sigma  # f_a = -V sigma g_a
    assert np.abs(out["force"] - expected).max() < 1e-6 * np.abs(expected).max()


def test_invertible_rotation_of_an_inverted_tet_is_proper():
    F = np.diag([1.0, 1.0, -0.5]) @ rotation(0.4, (1, 1, 0))
    R = po.rotation(po.F64, F, po.ROTATION_INVERTIBLE)
    assert abs(np.linalg.det(R) - 1.0) < 1e-12
    assert np.abs(R @ R.T - np.eye(3)).max() < 1e-12
    # U' V'^T with the smallest singular direction flipped
    U, s, Vt = np.linalg.svd(F)
    if np.linalg.det(U) < 0:
        U[:, 2] *= -1
    if np.linalg.det(Vt.T) < 0:
        Vt[2, :] *= -1
    assert np.abs(R - U @ Vt).max() < 1e-10


def test_polar_rotation_of_a_stretched_turn():
    R0 = rotation(0.9, (1, -2, 0.5))
    S = np.array([[1.2, 0.1, 0.0], [0.1, 0.9, 0.05], [0.0, 0.05, 1.1]])
    R = po.rotation(po.F64, R0 @ S, po.ROTATION_POLAR)
    assert np.abs(R - R0).max() < 1e-10


def plastic_case(eps, yield_stress=1e3, hardening=0.0, committed=None, margin=0.0):
    mat = po.material(1000.0, 1e6, 0.3, yield_stress=yield_stress, hardening=hardening)
    x = mapped(np.eye(3) + eps)
    return po.tet_point_trial(po.F64, x, REST, rest_inverse(), volume(), mat, committed, margin,
                              po.ROTATION_POLAR), mat


def test_point_inside_yield_surface_stays_elastic():
    eps = np.array([[1e-5, 0, 0], [0, 0, 0], [0, 0, 0]])
    out, _ = plastic_case(eps, yield_stress=1e5)
    assert out["yielding"] == 0 and out["loading"] == 0
    assert np.abs(out["plastic"]).max() == 0.0


@pytest.mark.parametrize("hardening", [0.0, 2e5])
def test_point_past_yield_returns_onto_the_surface(hardening):
    # pure shear strain, so the corotated strain equals eps
    g = 5e-3
    eps = np.array([[g, 0, 0], [0, -g, 0], [0, 0, 0]])
    out, mat = plastic_case(eps, yield_stress=1e3, hardening=hardening)
    lam, mu = lame(mat)
    assert out["yielding"] == 1
    dev = eps - np.trace(eps) / 3 * np.eye(3)
    q = math.sqrt(1.5) * np.linalg.norm(2 * mu * dev)
    gamma = (q - 1e3) / (3 * mu + hardening)
    assert abs(out["plastic"][9] - gamma) <= 1e-9 * gamma            # equivalent plastic strain
    ep = out["plastic"][:9].reshape(3, 3)
    assert abs(np.trace(ep)) < 1e-12                                  # plastic flow keeps volume
    after = 2 * mu * (dev - ep)
    q_after = math.sqrt(1.5) * np.linalg.norm(after)
    assert abs(q_after - (1e3 + hardening * gamma)) <= 1e-6 * q_after  # on the hardened surface


def test_consistent_tangent_matches_finite_differences_of_stress_response():
    # along a symmetric strain path with no rotation the element force derivative
    # is the algorithmic tangent (material.cc:636-650)
    g = 4e-3
    eps = np.array([[g, 1e-4, 0], [1e-4, -g, 0], [0, 0, 5e-4]])
    out, mat = plastic_case(eps, yield_stress=1e3, hardening=1e5, margin=0.0)
    assert out["loading"] == 1
    K = out["tangent"]
    x = mapped(np.eye(3) + eps)
    d = np.zeros((4, 3))
    d[1] = [1e-9, 0, 0]
    d[2] = [0, -1e-9, 0]
    plus = po.tet_point_trial(po.F64, x + d, REST, rest_inverse(), volume(), mat, None, 0.0, po.ROTATION_POLAR)
    minus = po.tet_point_trial(po.F64, x - d, REST, rest_inverse(), volume(), mat, None, 0.0, po.ROTATION_POLAR)
    fd = -(plus["force"] - minus["force"]).ravel() / 2.0
    assert np.abs(fd - K @ d.ravel()).max() <= 1e-3 * np.abs(K @ d.ravel()).max()


def test_free_fall_follows_the_generalized_alpha_recurrence():
    import talus_b200 as tb

    mesh = tb.box_mesh((2, 2, 2), voxel=0.1)
    mesh.anchored[:] = 0
    om = po.Mesh(mesh.rest_positions, mesh.node_mass, mesh.anchored, mesh.tet_nodes, mesh.rest_inverse,
                 mesh.volume, mesh.material)
    state = po.State.rest(om)
    settings = po.Settings(law=po.LAW_SNH, rigid_split=0, tolerance=1e-12, cg_iterations=200)
    rho = 0.5
    am, af = (2 * rho - 1) / (rho + 1), rho / (rho + 1)
    gamma, beta = 0.5 - am + af, 0.25 * (1 - am + af) ** 2
    h, g = 1.0 / 60.0, -9.81
    x, v, a = 0.0, 0.0, 0.0
    for _ in range(30):
        po.step(po.F64, om, state, [RUBBER], settings, (0.0, g, 0.0), h)
        a_new = (g - am * a) / (1 - am)       # (1 - am) a_{n+1} + am a_n = g
        x = x + h * v + h * h * ((0.5 - beta) * a + beta * a_new)
        v = v + h * ((1 - gamma) * a + gamma * a_new)
        a = a_new
    assert np.abs(state.position[:, 1] - mesh.rest_positions[:, 1] - x).max() <= 1e-9
    assert np.abs(state.velocity[:, 1] - v).max() <= 1e-9
    assert np.abs(state.position[:, [0, 2]] - mesh.rest_positions[:, [0, 2]]).max() <= 1e-12


def test_pinned_nodes_never_move_and_rest_stays_at_rest():
    import talus_b200 as tb

    mesh = tb.box_mesh((4, 4, 4), voxel=0.1, jitter=0.01, seed=3)
    om = po.Mesh(mesh.rest_positions, mesh.node_mass, mesh.anchored, mesh.tet_nodes, mesh.rest_inverse,
                 mesh.volume, mesh.material)
    state = po.State.rest(om)
    for _ in range(10):
        po.step(po.F64, om, state, [RUBBER], po.Settings(), (0.0, -9.81, 0.0), 1 / 60)
    pinned = mesh.anchored != 0
    assert np.array_equal(state.position[pinned], mesh.rest_positions[pinned])
    assert np.abs(state.position[~pinned] - mesh.rest_positions[~pinned]).max() > 1e-5
    still = po.State.rest(om)
    for _ in range(3):
        po.step(po.F64, om, still, [RUBBER], po.Settings(), (0.0, 0.0, 0.0), 1 / 60)
    assert np.abs(still.position - mesh.rest_positions).max() < 1e-14


def test_fp32_restatement_tracks_fp64_on_the_elastic_block():
    """The reference's own FP32 arithmetic against the FP64 oracle (a reported
    figure, not a bar): a few 1e-4 on the 8x8x8 block."""
    import talus_b200 as tb

    mesh = tb.box_mesh((8, 8, 8), voxel=0.1, jitter=0.01, seed=1)
    om = po.Mesh(mesh.rest_positions, mesh.node_mass, mesh.anchored, mesh.tet_nodes, mesh.rest_inverse,
                 mesh.volume, mesh.material)
    a, b = po.State.rest(om), po.State.rest(om)
    mat = [po.material(1000.0, 1e6, 0.3)]
    worst = 0.0
    for _ in range(10):
        po.step(po.F64, om, a, mat, po.Settings(), (0, -9.81, 0), 1 / 60)
        po.step(po.F32, om, b, mat, po.Settings(), (0, -9.81, 0), 1 / 60)
        scale = np.linalg.norm(a.position - mesh.rest_positions, axis=1).max()
        worst = max(worst, np.linalg.norm(b.position - a.position, axis=1).max() / scale)
    assert worst < 2e-3
