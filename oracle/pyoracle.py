"""ctypes binding of the CPU oracle (oracle/fem_oracle.cc).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py as the reference results.  The product package
``talus_b200`` never imports it.

The oracle restates talus::deformable::step (reference
src/talus/deformable/solver/solver.cc:3472-5901, contact block excluded) and
its tet laws (src/talus/deformable/material/material.cc).  Parity of the
restatement is pinned by the known-answer tests in tests/test_oracle_laws.py.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libfem_oracle.so")

F32, F64 = 0, 1
LAW_COROTATED, LAW_SNH = 0, 1
ROTATION_POLAR, ROTATION_INVERTIBLE = 0, 1
PLASTICITY_SMALL_STRAIN, PLASTICITY_HENCKY = 0, 1


class Material(C.Structure):
    _fields_ = [
        ("density", C.c_double),
        ("youngs_modulus", C.c_double),
        ("poissons_ratio", C.c_double),
        ("stiffness_damping", C.c_double),
        ("yield_stress", C.c_double),
        ("hardening_modulus", C.c_double),
        ("crush_stress", C.c_double),
        ("crush_limit", C.c_double),
        ("plastic_max", C.c_double),
    ]


class _Mesh(C.Structure):
    _fields_ = [
        ("nodes", C.c_uint32),
        ("tets", C.c_uint32),
        ("rest", C.c_void_p),
        ("node_mass", C.c_void_p),
        ("anchored", C.c_void_p),
        ("tet_nodes", C.c_void_p),
        ("rest_inverse", C.c_void_p),
        ("volume", C.c_void_p),
        ("lane", C.c_void_p),
        ("element_youngs", C.c_void_p),
        ("prescribed", C.c_void_p),
    ]


class _Settings(C.Structure):
    _fields_ = [
        ("substeps", C.c_uint32),
        ("cg_iterations", C.c_uint32),
        ("plastic_passes", C.c_uint32),
        ("law", C.c_uint32),
        ("tolerance", C.c_double),
        ("spectral_radius", C.c_double),
        ("rigid_split", C.c_uint32),
        ("plasticity", C.c_uint32),
    ]


class _State(C.Structure):
    _fields_ = [
        ("position", C.c_void_p),
        ("velocity", C.c_void_p),
        ("acceleration", C.c_void_p),
        ("rotation", C.c_void_p),
        ("plastic", C.c_void_p),
    ]


class Report(C.Structure):
    _fields_ = [
        ("substeps", C.c_uint32),
        ("cg_iterations", C.c_uint32),
        ("cg_capped_solves", C.c_uint32),
        ("plastic_evaluations", C.c_uint32),
        ("plastic_solves", C.c_uint32),
        ("plastic_backtracks", C.c_uint32),
        ("plastic_capped", C.c_uint32),
        ("plastic_linear_reads", C.c_uint32),
        ("plastic_handoffs", C.c_uint32),
        ("plastic_fallbacks", C.c_uint32),
        ("plastic_fallback_rejections", C.c_uint32),
        ("operator_applications", C.c_uint32),
        ("yielding", C.c_uint32),
        ("plastic_growth", C.c_uint32),
        ("non_finite", C.c_uint32),
        ("reserved", C.c_uint32),
        ("cg_worst_relative_residual", C.c_double),
        ("plastic_worst_residual", C.c_double),
        ("elastic_energy", C.c_double),
        ("kinetic_energy", C.c_double),
        ("seconds", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class SolverStats(C.Structure):
    """or_solver_stats: SolverStats (factor.h:28-38), the SystemFactor's size
    and the StepReport's factor counters."""
    _fields_ = [(n, C.c_uint32) for n in ("factor_age", "refactor_count", "retry_count", "substeps_since_refresh",
                                          "refresh_requested", "fresh_retry_failed")] + \
               [("mean_iterations", C.c_double), ("rows", C.c_uint32), ("ready", C.c_uint32),
                ("system_nonzeros", C.c_uint64), ("generation", C.c_uint64)] + \
               [(n, C.c_uint32) for n in ("refresh_requests", "refactors", "retries", "retries_failed",
                                          "wasted_iterations", "spent_before_refresh", "spent_after_refresh",
                                          "refreshed_at_age", "factor_applications", "reserved")]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class Solver:
    """A caller-held solver state (DeformableSolverState, factor.h:205-210)
    with its FP64 Cholesky factor; factor_budget is Settings::factorBudget."""

    def __init__(self, factor_budget: int = 32):
        self.handle = lib().or_solver_create(factor_budget)

    def stats(self) -> dict:
        out = SolverStats()
        lib().or_solver_get_stats(self.handle, C.byref(out))
        return out.as_dict()

    def close(self):
        if self.handle:
            lib().or_solver_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()


class _Grid(C.Structure):
    _fields_ = [
        ("cells", C.c_uint32 * 3),
        ("voxel", C.c_double),
        ("origin", C.c_double * 3),
        ("jitter", C.c_double),
        ("seed", C.c_uint64),
        ("density", C.c_double),
        ("anchor_axis", C.c_uint32),
        ("anchor_side", C.c_uint32),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run `make -C oracle`)")
        _lib = C.CDLL(LIB_PATH)
        _lib.or_grid_counts.argtypes = [C.POINTER(_Grid), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        _lib.or_grid_build.argtypes = [C.POINTER(_Grid)] + [C.c_void_p] * 8
        _lib.or_step.argtypes = [C.c_int, C.POINTER(_Mesh), C.POINTER(_State), C.POINTER(Material), C.c_uint32,
                                 C.POINTER(_Settings), C.c_void_p, C.c_double, C.POINTER(Report)]
        _lib.or_step_solver.argtypes = list(_lib.or_step.argtypes) + [C.c_void_p]
        _lib.or_solver_create.argtypes = [C.c_uint32]
        _lib.or_solver_create.restype = C.c_void_p
        _lib.or_solver_destroy.argtypes = [C.c_void_p]
        _lib.or_solver_destroy.restype = None
        _lib.or_solver_get_stats.argtypes = [C.c_void_p, C.POINTER(SolverStats)]
        _lib.or_tet_point_trial.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                            C.POINTER(Material), C.c_void_p, C.c_double, C.c_int, C.c_int,
                                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.or_tet_trial.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                      C.POINTER(Material), C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.or_snh_tet.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                    C.POINTER(Material), C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.or_rotation.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p]
        _lib.or_damping_apply.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                          C.POINTER(Material), C.c_void_p, C.c_void_p]
        _lib.or_hencky_return.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.or_hencky_von_mises.argtypes = [C.c_void_p, C.c_double]
        _lib.or_hencky_von_mises.restype = C.c_double
        _lib.or_hencky_flow.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double,
                                        C.POINTER(Material)]
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


def material(density=1000.0, youngs=1e6, poisson=0.3, damping=0.0, yield_stress=np.inf, hardening=0.0,
             crush_stress=np.inf, crush_limit=1.0, plastic_max=np.inf) -> Material:
    return Material(density, youngs, poisson, damping, yield_stress, hardening, crush_stress, crush_limit, plastic_max)


@dataclass
class Mesh:
    rest: np.ndarray            # [V,3] f64
    node_mass: np.ndarray       # [V] f64
    anchored: np.ndarray        # [V] u8
    tet_nodes: np.ndarray       # [T,4] u32
    rest_inverse: np.ndarray    # [T,3,3] f64 (row-major Dm^-1)
    volume: np.ndarray          # [T] f64
    lane: np.ndarray            # [T] u32
    grid_index: np.ndarray | None = None   # [V] u32 lattice sample index
    cells: tuple | None = None
    element_youngs: np.ndarray | None = None
    prescribed: np.ndarray | None = None   # [V,3] f64

    @property
    def nodes(self) -> int:
        return int(self.rest.shape[0])

    @property
    def tets(self) -> int:
        return int(self.tet_nodes.shape[0])

    def lattice(self) -> np.ndarray:
        """[V,3] integer lattice coordinates of each node."""
        rx, ry = self.cells[0] + 1, self.cells[1] + 1
        g = self.grid_index.astype(np.int64)
        return np.stack([g % rx, (g // rx) % ry, g // (rx * ry)], axis=1)


def build_grid(cells, voxel=0.1, origin=(0.0, 0.0, 0.0), jitter=0.0, seed=0, density=1000.0,
               anchor_axis=1, anchor_side=0) -> Mesh:
    g = _Grid((C.c_uint32 * 3)(*cells), voxel, (C.c_double * 3)(*origin), jitter, seed, density,
              anchor_axis, anchor_side)
    V, T = C.c_uint32(), C.c_uint32()
    if lib().or_grid_counts(C.byref(g), C.byref(V), C.byref(T)) != 0:
        raise ValueError("bad grid")
    V, T = V.value, T.value
    rest = np.zeros((V, 3)); mass = np.zeros(V); anchored = np.zeros(V, np.uint8)
    tet = np.zeros((T, 4), np.uint32); rinv = np.zeros((T, 3, 3)); vol = np.zeros(T)
    lane = np.zeros(T, np.uint32); gi = np.zeros(V, np.uint32)
    rc = lib().or_grid_build(C.byref(g), _ptr(rest), _ptr(mass), _ptr(anchored), _ptr(tet), _ptr(rinv),
                             _ptr(vol), _ptr(lane), _ptr(gi))
    if rc != 0:
        raise RuntimeError("or_grid_build failed")
    return Mesh(rest, mass, anchored, tet, rinv, vol, lane, gi, tuple(cells))


@dataclass
class State:
    position: np.ndarray
    velocity: np.ndarray
    acceleration: np.ndarray
    rotation: np.ndarray   # [T,3,3]
    plastic: np.ndarray    # [T,10]

    @staticmethod
    def rest(mesh: Mesh, hencky: bool = False) -> "State":
        """restState (solver.cc:2420-2453) at the identity pose; anchored nodes
        start with their prescribed velocity.  ``hencky``: the plastic slot holds
        the identity plastic map P = I and hardening 0."""
        v = np.zeros((mesh.nodes, 3))
        if mesh.prescribed is not None:
            v[mesh.anchored != 0] = mesh.prescribed[mesh.anchored != 0]
        plastic = np.zeros((mesh.tets, 10))
        if hencky:
            plastic[:, [0, 4, 8]] = 1.0
        return State(mesh.rest.copy(), v, np.zeros((mesh.nodes, 3)), np.tile(np.eye(3), (mesh.tets, 1, 1)), plastic)

    def copy(self) -> "State":
        return State(self.position.copy(), self.velocity.copy(), self.acceleration.copy(), self.rotation.copy(),
                     self.plastic.copy())


@dataclass
class Settings:
    substeps: int = 1
    cg_iterations: int = 64
    plastic_passes: int = 40
    law: int = LAW_COROTATED
    tolerance: float = 1e-3
    spectral_radius: float = 0.5
    rigid_split: int = 2
    plasticity: int = PLASTICITY_SMALL_STRAIN


def step(precision: int, mesh: Mesh, state: State, materials, settings: Settings, gravity=(0.0, -9.81, 0.0),
         dt=1.0 / 60.0, report: Report | None = None, solver: "Solver | None" = None) -> Report:
    for a in (state.position, state.velocity, state.acceleration, state.rotation, state.plastic):
        assert a.dtype == np.float64 and a.flags.c_contiguous
    m = _Mesh(mesh.nodes, mesh.tets, _ptr(mesh.rest), _ptr(mesh.node_mass), _ptr(mesh.anchored),
              _ptr(mesh.tet_nodes), _ptr(mesh.rest_inverse), _ptr(mesh.volume), _ptr(mesh.lane),
              _ptr(mesh.element_youngs), _ptr(mesh.prescribed))
    s = _State(_ptr(state.position), _ptr(state.velocity), _ptr(state.acceleration), _ptr(state.rotation),
               _ptr(state.plastic))
    mats = (Material * len(materials))(*materials)
    st = _Settings(settings.substeps, settings.cg_iterations, settings.plastic_passes, settings.law,
                   settings.tolerance, settings.spectral_radius, settings.rigid_split, settings.plasticity)
    g = np.asarray(gravity, dtype=np.float64)
    rep = report if report is not None else Report()
    rc = lib().or_step_solver(precision, C.byref(m), C.byref(s), mats, len(materials), C.byref(st), _ptr(g), dt,
                              C.byref(rep), solver.handle if solver is not None else None)
    if rc != 0:
        raise RuntimeError(f"or_step failed: {rc}")
    return rep


def tet_point_trial(precision, deformed, rest, rest_inverse, volume, mat, committed=None, margin=0.0,
                    rotation_mode=ROTATION_INVERTIBLE, return_mapping=True, tangent=True):
    deformed = np.ascontiguousarray(deformed, np.float64); rest = np.ascontiguousarray(rest, np.float64)
    rinv = np.ascontiguousarray(rest_inverse, np.float64)
    committed = np.zeros(10) if committed is None else np.ascontiguousarray(committed, np.float64)
    force = np.zeros((4, 3)); rot = np.zeros((3, 3)); plastic = np.zeros(10); scal = np.zeros(4)
    tan = np.zeros((12, 12)) if tangent else None
    lib().or_tet_point_trial(precision, _ptr(deformed), _ptr(rest), _ptr(rinv), volume, C.byref(mat),
                             _ptr(committed), margin, rotation_mode, int(return_mapping), _ptr(force), _ptr(rot),
                             _ptr(plastic), _ptr(tan), _ptr(scal))
    return dict(force=force, rotation=rot, plastic=plastic, tangent=tan, energy=scal[0], plastic_work=scal[1],
                yielding=int(scal[2]), loading=int(scal[3]))


def tet_trial(precision, deformed, rest, rest_inverse, volume, mat, rotation_mode=ROTATION_INVERTIBLE):
    deformed = np.ascontiguousarray(deformed, np.float64); rest = np.ascontiguousarray(rest, np.float64)
    rinv = np.ascontiguousarray(rest_inverse, np.float64)
    force = np.zeros((4, 3)); rot = np.zeros((3, 3)); energy = np.zeros(1)
    lib().or_tet_trial(precision, _ptr(deformed), _ptr(rest), _ptr(rinv), volume, C.byref(mat), rotation_mode,
                       _ptr(force), _ptr(rot), _ptr(energy))
    return dict(force=force, rotation=rot, energy=energy[0])


def snh_tet(precision, deformed, rest, rest_inverse, volume, mat):
    deformed = np.ascontiguousarray(deformed, np.float64); rest = np.ascontiguousarray(rest, np.float64)
    rinv = np.ascontiguousarray(rest_inverse, np.float64)
    force = np.zeros((4, 3)); energy = np.zeros(1); hess = np.zeros((12, 12))
    lib().or_snh_tet(precision, _ptr(deformed), _ptr(rest), _ptr(rinv), volume, C.byref(mat), _ptr(force),
                     _ptr(energy), _ptr(hess))
    return dict(force=force, energy=energy[0], hessian=hess)


def damping_apply(precision, corners, rotation, rest_inverse, volume, mat, direction):
    """D(direction) of one tet with its rigid fit at `corners` (factor.cc:843-853)."""
    a = [np.ascontiguousarray(x, np.float64) for x in (corners, rotation, rest_inverse, direction)]
    out = np.zeros((4, 3))
    lib().or_damping_apply(precision, _ptr(a[0]), _ptr(a[1]), _ptr(a[2]), volume, C.byref(mat), _ptr(a[3]), _ptr(out))
    return out


def rotation(precision, gradient, mode=ROTATION_INVERTIBLE):
    g = np.ascontiguousarray(gradient, np.float64); out = np.zeros((3, 3))
    lib().or_rotation(precision, _ptr(g), mode, _ptr(out))
    return out


def hencky_return(elastic, shear, yield_stress):
    """plasticflow.cc:110-150 returnMap of one point: None inside the yield
    surface, else (returned elastic map, strain, trial stress)."""
    fe = np.ascontiguousarray(elastic, np.float64)
    out = np.zeros((3, 3)); strain = np.zeros(1); trial = np.zeros(1)
    if not lib().or_hencky_return(_ptr(fe), shear, yield_stress, _ptr(out), _ptr(strain), _ptr(trial)):
        return None
    return out, float(strain[0]), float(trial[0])


def hencky_von_mises(elastic, shear) -> float:
    """plasticflow.cc:96-108 vonMises."""
    return float(lib().or_hencky_von_mises(_ptr(np.ascontiguousarray(elastic, np.float64)), shear))


def hencky_flow(deformation, plastic, hardening, shear, bulk, mat: Material):
    """plasticflow.cc:184-247 flowLattice at one point with the material's
    yield stress, hardening, crush and plastic cap: (changed, P, hardening)."""
    f = np.ascontiguousarray(deformation, np.float64)
    p = np.array(plastic, np.float64, order="C")
    h = np.array([hardening], np.float64)
    changed = lib().or_hencky_flow(_ptr(f), _ptr(p), _ptr(h), shear, bulk, C.byref(mat))
    return bool(changed), p, float(h[0])
