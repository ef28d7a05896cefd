"""Gradient-check harness of the differentiable rollout.

The rollout (talus_b200.rollout, C ABI tl_rollout_*) is wrapped in a
torch.autograd.Function here, and only here: torch is the harness, the
gradients come from the library's hand-written adjoint.

Problem (the differentiable-rollout workload): a cells^3 block of 0.1 m
cubes (6 Kuhn tets each), neo-Hookean, E0 = 1e6 Pa, nu = 0.3, rho = 1000,
base anchored, gravity, dt = 1/60.  The target is the final position of a
rollout whose per-element E is E0 exp(0.3 N(0, 1)) (seeded); the loss is
L(E, v0) = |x_T(E, v0) - x_target|^2.  Gradients with respect to per-element
E and initial velocity v0 are compared with FP64 central finite differences
of the same GPU forward, step h = 1e-6 relative, along random directions and
for single elements.

    python -m talus_b200.gradcheck --cells 16 --steps 30
"""
from __future__ import annotations

import argparse
import json
import math
import sys

import numpy as np


def make_problem(cells=16, steps=30, seed=7, precision=None, checkpoint_every=5, newton_reads=4, tolerance=1e-10,
                 context=None):
    import talus_b200 as tb

    precision = tb.FP64 if precision is None else precision
    mesh = tb.box_mesh((cells, cells, cells), voxel=0.1, seed=seed)
    mat = tb.PhysicalMaterial(density=1000.0, youngs_modulus=1.0e6, poissons_ratio=0.3)
    system = tb.System(mesh, [mat], precision, context)
    rng = np.random.default_rng(seed)
    e_target = 1.0e6 * np.exp(0.3 * rng.standard_normal(mesh.tets))
    settings = tb.rollout.converged_settings(tolerance=tolerance)
    roll = tb.Rollout(system, steps, checkpoint_every=checkpoint_every, newton_reads=newton_reads,
                      settings=settings)
    prob = Problem(mesh, system, roll, np.full(mesh.tets, 1.0e6), np.zeros((mesh.nodes, 3)))
    prob.target = prob.final_position(e_target, prob.v0)
    prob.e_target = e_target
    return prob


class Problem:
    def __init__(self, mesh, system, roll, youngs, v0):
        self.mesh, self.system, self.roll = mesh, system, roll
        self.youngs, self.v0 = youngs, v0
        self.target = None

    def final_position(self, youngs, v0):
        import talus_b200 as tb

        self.system.set_youngs(youngs)
        state = tb.rest_state(self.mesh)
        state.velocity[...] = v0
        state.velocity[self.mesh.anchored != 0] = 0.0
        self.system.set_state(state)
        self.roll.forward()
        return self.system.get_state().position

    def close(self):
        self.roll.close()
        self.system.close()

    def loss(self, youngs, v0):
        d = self.final_position(youngs, v0) - self.target
        return float(np.sum(d * d))

    def gradients(self, youngs, v0):
        d = self.final_position(youngs, v0) - self.target
        g = self.roll.adjoint(2.0 * d)
        return float(np.sum(d * d)), g


def autograd_function():
    """torch.autograd.Function over the rollout: (E, v0) -> x_T, backward by
    tl_rollout_adjoint.  Tensors are CPU float64 (the C ABI's host buffers)."""
    import torch

    class RolloutFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, youngs, v0, problem):
            x = problem.final_position(youngs.detach().numpy(), v0.detach().numpy())
            ctx.problem = problem
            return torch.from_numpy(x.copy())

        @staticmethod
        def backward(ctx, grad_x):
            g = ctx.problem.roll.adjoint(grad_x.detach().numpy())
            return torch.from_numpy(g.youngs.copy()), torch.from_numpy(g.velocity.copy()), None

    return RolloutFunction


def torch_loss_and_grad(problem, youngs, v0):
    """Loss and gradients through torch autograd (the harness path)."""
    import torch

    fn = autograd_function()
    e = torch.tensor(youngs, dtype=torch.float64, requires_grad=True)
    v = torch.tensor(v0, dtype=torch.float64, requires_grad=True)
    x = fn.apply(e, v, problem)
    loss = ((x - torch.from_numpy(problem.target)) ** 2).sum()
    loss.backward()
    return float(loss.detach()), e.grad.numpy(), v.grad.numpy()


def central_difference(f, h):
    return (f(h) - f(-h)) / (2.0 * h)


def check(problem, directions=3, elements=3, seed=11, h=1e-6):
    """Directional and per-element FD checks; returns a report dict."""
    rng = np.random.default_rng(seed)
    youngs, v0 = problem.youngs, problem.v0
    loss, ge, gv = torch_loss_and_grad(problem, youngs, v0)
    out = {"loss": loss, "tets": problem.mesh.tets, "nodes": problem.mesh.nodes, "checks": []}
    free = (problem.mesh.anchored == 0)[:, None]
    vscale = 9.81 * problem.roll.steps / 60.0  # free-fall speed over the rollout
    for k in range(directions):
        r = rng.standard_normal(youngs.shape)
        fd = central_difference(lambda t: problem.loss(youngs * (1.0 + t * r), v0), h)
        ad = float(np.sum(ge * youngs * r))
        out["checks"].append({"kind": "E direction", "fd": fd, "adjoint": ad, "rel": abs(ad - fd) / abs(fd)})
        d = rng.standard_normal(v0.shape) * free
        fd = central_difference(lambda t: problem.loss(youngs, v0 + t * vscale * d), h)
        ad = float(np.sum(gv * vscale * d))
        out["checks"].append({"kind": "v0 direction", "fd": fd, "adjoint": ad, "rel": abs(ad - fd) / abs(fd)})
    order = np.argsort(-np.abs(ge * youngs))
    for e in order[:elements]:
        unit = np.zeros_like(youngs)
        unit[e] = 1.0
        fd = central_difference(lambda t: problem.loss(youngs * (1.0 + t * unit), v0), h)
        ad = float(ge[e] * youngs[e])
        out["checks"].append({"kind": f"E[{int(e)}]", "fd": fd, "adjoint": ad, "rel": abs(ad - fd) / abs(fd)})
    out["worst_rel"] = max(c["rel"] for c in out["checks"])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cells", type=int, default=16)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--checkpoint-every", type=int, default=5)
    ap.add_argument("--directions", type=int, default=3)
    ap.add_argument("--elements", type=int, default=3)
    args = ap.parse_args()
    prob = make_problem(args.cells, args.steps, checkpoint_every=args.checkpoint_every)
    rep = check(prob, args.directions, args.elements)
    print(json.dumps(rep))
    return 0 if rep["worst_rel"] < 1e-4 and math.isfinite(rep["worst_rel"]) else 1


if __name__ == "__main__":
    sys.exit(main())
