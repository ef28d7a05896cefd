"""Host mirror of talus::deformable's tet-step interface over the C ABI.

Names and argument meaning follow the reference
(src/talus/mesh.h, src/talus/material.h,
src/talus/deformable/solver/solver.h):

* ``PhysicalMaterial``  -- talus::PhysicalMaterial (material.h:12-29)
* ``PreparedMesh``      -- the tet fields of talus::PreparedMesh (mesh.h:25-44)
* ``DeformableState``   -- talus::DeformableState (mesh.h:56-62)
* ``Settings``          -- the non-contact fields of deformable::Settings (solver.h:51-107)
* ``StepReport``        -- the non-contact counters of deformable::StepReport (solver.h:211-311)
* ``step``              -- deformable::step (solver.h:451-462) with no contacts,
                           no rigid partners and no DeformableSolverState
* ``rest_state``        -- deformable::restState (solver.h:331-334) at the identity pose

Every call runs the CUDA kernels of libtalus_fem.so; nothing here computes
physics.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _capi as capi
from ._capi import check

FP64 = capi.TL_FP64
FP32_MIXED = capi.TL_FP32_MIXED
COROTATED = capi.TL_LAW_COROTATED
NEO_HOOKEAN = capi.TL_LAW_SNH


@dataclass
class PhysicalMaterial:
    density: float = 1000.0
    youngs_modulus: float = 0.0
    poissons_ratio: float = 0.3
    stiffness_damping: float = 0.0
    yield_stress: float = math.inf
    hardening_modulus: float = 0.0
    # finite-strain flow only (System.set_plasticity("hencky")); applied per
    # lane through tl_system_set_flow_limits, not part of tl_material
    crush_stress: float = math.inf
    crush_limit: float = 1.0
    plastic_max: float = math.inf

    def _c(self) -> capi.tl_material:
        return capi.tl_material(self.density, self.youngs_modulus, self.poissons_ratio, self.stiffness_damping,
                                self.yield_stress, self.hardening_modulus)


@dataclass
class PreparedMesh:
    rest_positions: np.ndarray          # [V,3] float64
    node_mass: np.ndarray               # [V]
    anchored: np.ndarray                # [V] uint8
    tet_nodes: np.ndarray               # [T,4] uint32
    rest_inverse: np.ndarray            # [T,3,3] row-major Dm^-1
    volume: np.ndarray                  # [T]
    material: np.ndarray                # [T] uint32 lane
    prescribed_velocity: np.ndarray | None = None   # [V,3] velocity of anchored nodes
    element_youngs: np.ndarray | None = None        # [T] per-element E
    lattice: np.ndarray | None = None               # [V,3] lattice coordinates (generator output)
    cells: tuple | None = None

    @property
    def nodes(self) -> int:
        return int(self.rest_positions.shape[0])

    @property
    def tets(self) -> int:
        return int(self.tet_nodes.shape[0])

    def face(self, axis: int, side: int) -> np.ndarray:
        """Boolean mask of the nodes on one face of a generated box."""
        value = 0 if side == 0 else self.cells[axis]
        return self.lattice[:, axis] == value


@dataclass
class DeformableState:
    position: np.ndarray      # [V,3]
    velocity: np.ndarray      # [V,3]
    acceleration: np.ndarray  # [V,3]
    rotation: np.ndarray      # [T,3,3] CommittedTet::rotation
    plastic: np.ndarray       # [T,10] PlasticPoint: strain (row-major 3x3), equivalent

    def copy(self) -> "DeformableState":
        return DeformableState(self.position.copy(), self.velocity.copy(), self.acceleration.copy(),
                               self.rotation.copy(), self.plastic.copy())


def rest_state(mesh: PreparedMesh, hencky: bool = False) -> DeformableState:
    """restState (solver.cc:2420-2453) at the identity pose.  Anchored nodes with
    a prescribed velocity start moving with it.  ``hencky``: the plastic slot
    holds the identity plastic map (P = I, hardening 0) that the finite-strain
    flow starts from, instead of a zero plastic strain."""
    velocity = np.zeros((mesh.nodes, 3))
    if mesh.prescribed_velocity is not None:
        held = mesh.anchored != 0
        velocity[held] = mesh.prescribed_velocity[held]
    plastic = np.zeros((mesh.tets, 10))
    if hencky:
        plastic[:, [0, 4, 8]] = 1.0
    return DeformableState(mesh.rest_positions.astype(np.float64).copy(), velocity, np.zeros((mesh.nodes, 3)),
                           np.tile(np.eye(3), (mesh.tets, 1, 1)), plastic)


@dataclass
class Settings:
    substeps: int = 1
    cg_iterations: int = 64
    plastic_passes: int = 40
    tolerance: float = 1.0e-3
    spectral_radius: float = 0.5
    rigid_split: int = capi.TL_RIGID_SPLIT_PROJECTED
    law: int = COROTATED
    profile: bool = False   # TL_FLAG_PROFILE: per-kernel-class device times in the report
    trace: bool = False     # TL_FLAG_TRACE: record each PCG launch's iterations (System.trace)

    def _c(self) -> capi.tl_settings:
        flags = (capi.TL_FLAG_PROFILE if self.profile else 0) | (capi.TL_FLAG_TRACE if self.trace else 0)
        return capi.tl_settings(self.substeps, self.cg_iterations, self.plastic_passes, self.rigid_split, self.law,
                                flags, self.tolerance, self.spectral_radius)


class StepReport(capi.tl_step_report):
    """Accumulated like the reference's StepReport (solver.cc:3612-3615)."""


def _ptr(a):
    return None if a is None else a.ctypes.data


class Context:
    """One CUDA device + stream (tl_ctx)."""

    def __init__(self, device: int = 0):
        handle = C.c_void_p()
        status = capi.lib().tl_ctx_create(device, C.byref(handle))
        if status != capi.TL_OK:
            raise capi.TalusError(status, "tl_ctx_create")
        self.handle = handle

    def pin(self, array):
        """Page-locks a contiguous numpy array (tl_host_register), so state
        crosses to and from it by one DMA instead of the library's staging."""
        check(capi.lib().tl_host_register(self.handle, array.ctypes.data, array.nbytes), self.handle)

    def unpin(self, array):
        check(capi.lib().tl_host_unregister(self.handle, array.ctypes.data), self.handle)

    def close(self):
        if self.handle:
            capi.lib().tl_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_context: Context | None = None


def default_context() -> Context:
    global _default_context
    if _default_context is None:
        _default_context = Context(0)
    return _default_context


class _Body:
    """Keeps a mesh's arrays alive in the layout the C ABI reads."""

    def __init__(self, mesh: PreparedMesh, materials):
        self.rest = np.ascontiguousarray(mesh.rest_positions, np.float64)
        self.mass = np.ascontiguousarray(mesh.node_mass, np.float64)
        self.anchored = np.ascontiguousarray(mesh.anchored, np.uint8)
        self.tets = np.ascontiguousarray(mesh.tet_nodes, np.uint32)
        self.rinv = np.ascontiguousarray(mesh.rest_inverse, np.float64)
        self.volume = np.ascontiguousarray(mesh.volume, np.float64)
        self.lane = np.ascontiguousarray(mesh.material, np.uint32)
        self.youngs = None if mesh.element_youngs is None else np.ascontiguousarray(mesh.element_youngs, np.float64)
        self.pres = None if mesh.prescribed_velocity is None else np.ascontiguousarray(mesh.prescribed_velocity,
                                                                                       np.float64)
        self.mats = (capi.tl_material * max(1, len(materials)))(*[m._c() for m in materials])
        self.lanes = len(materials)
        self.desc = capi.tl_mesh_desc(mesh.nodes, mesh.tets, _ptr(self.rest), _ptr(self.mass), _ptr(self.anchored),
                                      _ptr(self.tets), _ptr(self.rinv), _ptr(self.volume), _ptr(self.lane),
                                      self.mats, self.lanes, _ptr(self.youngs), _ptr(self.pres))


class System:
    """Bodies resident in device memory (tl_system).  ``count > 1`` bodies are
    stepped together (the batched form)."""

    def __init__(self, meshes, materials, precision: int = FP64, context: Context | None = None):
        if isinstance(meshes, PreparedMesh):
            meshes = [meshes]
        if materials and isinstance(materials[0], PhysicalMaterial):
            materials = [materials] * len(meshes)
        self.context = context or default_context()
        self.precision = precision
        self.meshes = list(meshes)
        self._bodies = [_Body(m, mats) for m, mats in zip(self.meshes, materials)]
        descs = (capi.tl_mesh_desc * len(self._bodies))(*[b.desc for b in self._bodies])
        handle = C.c_void_p()
        check(capi.lib().tl_system_create(self.context.handle, descs, len(self._bodies), precision,
                                          C.byref(handle)), self.context.handle)
        self.handle = handle
        default = (math.inf, 1.0, math.inf)
        for b, mats in enumerate(materials):
            for lane, m in enumerate(mats):
                limits = (m.crush_stress, m.crush_limit, m.plastic_max)
                if limits != default:
                    check(capi.lib().tl_system_set_flow_limits(handle, b, lane, *limits), self.context.handle)

    def close(self):
        if getattr(self, "handle", None):
            capi.lib().tl_system_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, state: DeformableState, body: int = 0):
        arrs = [np.ascontiguousarray(a, np.float64) for a in
                (state.position, state.velocity, state.acceleration, state.rotation, state.plastic)]
        check(capi.lib().tl_state_set(self.handle, body, capi.TL_DTYPE_F64, *[_ptr(a) for a in arrs]),
              self.context.handle)

    def get_state(self, body: int = 0) -> DeformableState:
        m = self.meshes[body]
        out = DeformableState(np.zeros((m.nodes, 3)), np.zeros((m.nodes, 3)), np.zeros((m.nodes, 3)),
                              np.zeros((m.tets, 3, 3)), np.zeros((m.tets, 10)))
        check(capi.lib().tl_state_get(self.handle, body, capi.TL_DTYPE_F64, _ptr(out.position), _ptr(out.velocity),
                                      _ptr(out.acceleration), _ptr(out.rotation), _ptr(out.plastic)),
              self.context.handle)
        return out

    def evaluate(self, settings: Settings, body: int = 0):
        """Internal node forces [V,3] and per-tet yield flags [T] at the
        positions the body holds (tl_evaluate); no state changes."""
        m = self.meshes[body]
        forces = np.zeros((m.nodes, 3))
        flags = np.zeros(m.tets, np.uint8)
        check(capi.lib().tl_evaluate(self.handle, body, C.byref(settings._c()), _ptr(forces), _ptr(flags)),
              self.context.handle)
        return forces, flags

    def set_youngs(self, youngs, body: int = 0):
        """Per-element Young's modulus of one body (tl_system_set_youngs)."""
        e = np.ascontiguousarray(youngs, np.float64)
        if e.shape != (self.meshes[body].tets,):
            raise ValueError("one modulus per tet")
        check(capi.lib().tl_system_set_youngs(self.handle, body, _ptr(e)), self.context.handle)

    def tune(self, pcg_blocks_per_sm: int = 0, graph: bool = True):
        """Launch shape (tl_system_tune): cap on persistent-PCG blocks per SM
        (0 = occupancy limit) and CUDA-graph replay of batched elastic steps."""
        check(capi.lib().tl_system_tune(self.handle, int(pcg_blocks_per_sm), 1 if graph else 0), self.context.handle)

    def tune_shape(self, row_group: int = 0, batch_blocks: int = 0):
        """Launch shape of the assembled-operator PCG (tl_system_tune_shape):
        column slots per round trip of a matrix row (2 or 4, 0 = default) and
        resident blocks per SM of the batched kernels (3 or 4, 0 = 4).  The
        results are bitwise the same for every shape."""
        check(capi.lib().tl_system_tune_shape(self.handle, capi.TL_SHAPE_ROW_GROUP, int(row_group)), self.context.handle)
        check(capi.lib().tl_system_tune_shape(self.handle, capi.TL_SHAPE_BATCH_BLOCKS, int(batch_blocks)),
              self.context.handle)

    def use_factor(self, enable: bool = True, factor_budget: int = 32):
        """Hold a solver state for this one-body system (tl_system_use_factor;
        the DeformableSolverState* of deformable::step): its PCG is then
        preconditioned by the FP64 Cholesky factor of the system, refreshed as
        the reference refreshes it.  factor_budget is Settings::factorBudget."""
        check(capi.lib().tl_system_use_factor(self.handle, 1 if enable else 0, int(factor_budget)),
              self.context.handle)

    def factor_stats(self) -> dict:
        """SolverStats, factor size and factor counters (tl_system_factor_stats)."""
        out = capi.tl_factor_stats()
        check(capi.lib().tl_system_factor_stats(self.handle, C.byref(out)), self.context.handle)
        return out.as_dict()

    def set_solver(self, form: str = "auto"):
        """PCG operator form of a system (tl_system_set_solver): "auto",
        "assembled" (3x3 node blocks assembled once per solve),
        "assembled-two-phase" / "assembled-pipelined" (the same matrix, a batch
        iterating with two grid barriers per iteration or with one) or
        "elementwise" (applied element by element every iteration)."""
        code = {"auto": capi.TL_SOLVER_AUTO, "assembled": capi.TL_SOLVER_ASSEMBLED,
                "assembled-two-phase": capi.TL_SOLVER_ASSEMBLED_TWO_PHASE,
                "assembled-pipelined": capi.TL_SOLVER_ASSEMBLED_PIPELINED,
                "elementwise": capi.TL_SOLVER_ELEMENTWISE}[form]
        check(capi.lib().tl_system_set_solver(self.handle, code), self.context.handle)

    def set_plasticity(self, mode: str = "small_strain"):
        """Plasticity of the yielding lanes (tl_system_set_plasticity):
        "small_strain" (the tet law's J2 return inside the step) or "hencky"
        (finite-strain flow after each step from a per-tet plastic rest
        shape; the state's plastic slot then holds P = Fp^-1 row-major and
        the hardening variable).  Resets every tet to P = I, hardening 0."""
        code = {"small_strain": capi.TL_PLASTICITY_SMALL_STRAIN, "hencky": capi.TL_PLASTICITY_HENCKY}[mode]
        check(capi.lib().tl_system_set_plasticity(self.handle, code), self.context.handle)

    def trace(self) -> list:
        """Iterations of every PCG launch made with Settings.trace, oldest first."""
        count = C.c_uint32()
        check(capi.lib().tl_system_trace(self.handle, None, 0, C.byref(count)), self.context.handle)
        out = np.zeros(max(1, count.value), np.uint32)
        check(capi.lib().tl_system_trace(self.handle, out.ctypes.data, count.value, C.byref(count)),
              self.context.handle)
        return out[:count.value].tolist()

    def substeps(self, body: int = 0):
        """The last step's per-substep solve records of one body
        (tl_step_substeps): PCG iterations, starting and final relative
        residuals, like StepReport::cgPerSubstep / cgStartResidual /
        cgEndResidual (solver.h:299-301)."""
        count = C.c_uint32()
        it = np.zeros(16, np.uint32)
        start = np.zeros(16)
        end = np.zeros(16)
        check(capi.lib().tl_step_substeps(self.handle, body, it.ctypes.data, start.ctypes.data, end.ctypes.data, 16,
                                          C.byref(count)), self.context.handle)
        k = min(16, count.value)
        return it[:k].tolist(), start[:k].tolist(), end[:k].tolist()

    def step(self, settings: Settings, gravity=(0.0, -9.81, 0.0), delta_time: float = 1.0 / 60.0, reports=None):
        """One deformable::step of every body; returns the per-body reports
        (accumulated into ``reports`` when given).  A non-finite state is
        reported (report.non_finite), not raised, like the reference."""
        if reports is None:
            reports = (StepReport * len(self._bodies))()
        g = np.asarray(gravity, np.float64)
        status = capi.lib().tl_step(self.handle, C.byref(settings._c()), _ptr(g), float(delta_time), reports)
        if status not in (capi.TL_OK, capi.TL_ERR_NONFINITE):
            check(status, self.context.handle)
        return reports


_cache: dict = {}


def step(mesh: PreparedMesh, state: DeformableState, materials, settings: Settings, gravity, delta_time: float,
         report: StepReport | None = None, precision: int = FP64) -> StepReport:
    """talus::deformable::step(mesh, state, materials, settings, gravity, deltaTime,
    {}, {}, nullptr, report): advances ``state`` in place on the GPU."""
    key = (id(mesh), precision, tuple((m.density, m.youngs_modulus, m.poissons_ratio, m.stiffness_damping,
                                       m.yield_stress, m.hardening_modulus) for m in materials))
    system = _cache.get(key)
    if system is None:
        system = System(mesh, list(materials), precision)
        _cache[key] = system
    system.set_state(state)
    report = report if report is not None else StepReport()
    reports = (StepReport * 1)(report)
    system.step(settings, gravity, delta_time, reports)
    C.memmove(C.addressof(report), C.addressof(reports[0]), C.sizeof(StepReport))
    got = system.get_state()
    state.position[...] = got.position
    state.velocity[...] = got.velocity
    state.acceleration[...] = got.acceleration
    state.rotation[...] = got.rotation
    state.plastic[...] = got.plastic
    return report
