"""Differentiable rollout of the elastic step over the C ABI
(tl_rollout_create / forward / adjoint, include/talus_fem.h).

    system = tb.System(mesh, [material], tb.FP64)
    system.set_state(tb.rest_state(mesh))
    roll = Rollout(system, steps=30, checkpoint_every=5)
    roll.forward()                       # system now holds x_T
    grads = roll.adjoint(dl_dx_final)    # dL/dE per tet, dL/dv0, dL/dx0

The forward is `steps` implicit steps with the neo-Hookean law, each solved
by `newton_reads` linearised reads at the settings' PCG tolerance; the adjoint
differentiates the converged step (implicit-function theorem), recomputing
each checkpoint segment on the device.  Nothing here computes physics.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _capi as capi
from ._capi import check
from .deformable import NEO_HOOKEAN, Settings, StepReport, System


@dataclass
class Gradients:
    youngs: np.ndarray          # dL/dE [T]
    velocity: np.ndarray        # dL/dv0 [V,3]
    position: np.ndarray        # dL/dx0 [V,3]
    seconds: float              # device time of the adjoint (recomputation included)


def converged_settings(tolerance: float = 1e-10, cg_iterations: int = 4000) -> Settings:
    """Settings of a differentiable rollout: the neo-Hookean law and a PCG
    tolerance tight enough that each step's implicit equation is solved."""
    return Settings(law=NEO_HOOKEAN, cg_iterations=cg_iterations, tolerance=tolerance)


class Rollout:
    def __init__(self, system: System, steps: int, checkpoint_every: int = 5, newton_reads: int = 4,
                 settings: Settings | None = None, gravity=(0.0, -9.81, 0.0), delta_time: float = 1.0 / 60.0):
        self.system = system
        self.settings = settings or converged_settings()
        desc = capi.tl_rollout_desc(steps, checkpoint_every, newton_reads, 0, float(delta_time),
                                    (C.c_double * 3)(*[float(g) for g in gravity]))
        handle = C.c_void_p()
        check(capi.lib().tl_rollout_create(system.handle, C.byref(desc), C.byref(self.settings._c()),
                                           C.byref(handle)), system.context.handle)
        self.handle = handle
        self.steps = steps
        self.forward_seconds = 0.0

    def close(self):
        if getattr(self, "handle", None):
            capi.lib().tl_rollout_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _live(self):
        if not getattr(self, "handle", None) or not getattr(self.system, "handle", None):
            raise RuntimeError("rollout or its system is closed")

    def forward(self) -> StepReport:
        """Runs the rollout from the system's current state (which it advances)."""
        self._live()
        report = StepReport()
        secs = C.c_double()
        check(capi.lib().tl_rollout_forward(self.handle, C.byref(report), C.byref(secs)),
              self.system.context.handle)
        self.forward_seconds = secs.value
        return report

    def adjoint(self, dl_dx_final, dl_dv_final=None) -> Gradients:
        self._live()
        mesh = self.system.meshes[0]
        dx = np.ascontiguousarray(dl_dx_final, np.float64).reshape(mesh.nodes, 3)
        dv = None if dl_dv_final is None else np.ascontiguousarray(dl_dv_final, np.float64).reshape(mesh.nodes, 3)
        ge = np.zeros(mesh.tets)
        gv = np.zeros((mesh.nodes, 3))
        gx = np.zeros((mesh.nodes, 3))
        secs = C.c_double()
        check(capi.lib().tl_rollout_adjoint(self.handle, dx.ctypes.data, None if dv is None else dv.ctypes.data,
                                            ge.ctypes.data, gv.ctypes.data, gx.ctypes.data, C.byref(secs)),
              self.system.context.handle)
        return Gradients(ge, gv, gx, secs.value)
