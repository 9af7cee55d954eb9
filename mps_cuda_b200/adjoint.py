"""Gradients of an MPS rollout: the hand-written adjoint behind torch.autograd.Function.

``rollout(nu, vel0, problem)`` advances a dam-break scene ``problem.steps`` steps from the
initial fluid velocities ``vel0`` at kinematic viscosity ``nu`` and returns the final fluid
positions and velocities. Its backward runs ``mps_adjoint_backward``: the device recomputes
each ``problem.every``-step segment from its checkpoint and applies the step adjoints in
reverse. Losses are plain torch code on the returned tensors, e.g. :func:`dambreak_loss`.

The reference (frsykzk/MPS_CUDA) has no derivative of its step; the forward here is the
same step as ``mps_step`` (kernel.cu:1904-1935), so the gradient is that of the reference's
method with every discrete choice of each step held fixed.
"""
from __future__ import annotations

import copy
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .solver import MPS, SceneDesc, dambreak, dambreak_params


@dataclass
class RolloutProblem:
    """A scene, its parameters and the rollout length. ``precision`` is an MPS_* code."""
    desc: SceneDesc
    dt: float
    steps: int
    every: int = 20
    precision: int = L.F64

    def __post_init__(self):
        sc = dambreak(self.desc)
        self.typ = sc["typ"]
        self.pos = sc["pos"]
        self.vel = sc["vel"]
        self.nrm = sc["nrm"]
        self.fluid = np.nonzero(self.typ == L.FLD)[0]
        self.params = dambreak_params(self.desc, dt=self.dt, precision=self.precision)

    def solver(self, nu: float, vel0: np.ndarray) -> MPS:
        """A handle at the initial state with viscosity nu and fluid velocities vel0 (3, nF)."""
        p = copy.copy(self.params)
        p.knm_vsc = float(nu)
        vel = self.vel.copy()
        vel[:, self.fluid] = vel0
        rd = np.float64 if self.precision == L.F64 else np.float32
        return MPS(p, self.typ, self.pos.astype(rd), vel.astype(rd), self.nrm.astype(rd))

    def run(self, nu: float, vel0: np.ndarray) -> dict:
        """Forward only: the final state of the rollout."""
        h = self.solver(nu, vel0)
        try:
            h.step(self.steps)
            return h.state()
        finally:
            h.close()


def _rollout_cls():
    import torch

    class Rollout(torch.autograd.Function):
        """(nu, vel0) -> (fluid positions, fluid velocities, alive mask) after the rollout."""

        @staticmethod
        def forward(ctx, nu, vel0, problem: RolloutProblem):
            v0 = vel0.detach().to("cpu", torch.float64).numpy()
            h = problem.solver(float(nu), v0)
            try:
                h.adjoint_record(problem.steps, problem.every)
                st = h.state()
            except Exception:
                h.close()
                raise
            ctx.h = h
            ctx.problem = problem
            f = problem.fluid
            pos = torch.from_numpy(np.ascontiguousarray(st["pos"][:, f], np.float64))
            vel = torch.from_numpy(np.ascontiguousarray(st["vel"][:, f], np.float64))
            alive = torch.from_numpy(st["typ"][f] == L.FLD)
            ctx.mark_non_differentiable(alive)
            dev = vel0.device
            return pos.to(dev), vel.to(dev), alive.to(dev)

        @staticmethod
        def backward(ctx, gpos, gvel, _galive):
            problem, h = ctx.problem, ctx.h
            n, f = problem.typ.shape[0], problem.fluid
            lam_pos = np.zeros((3, n))
            lam_vel = np.zeros((3, n))
            if gpos is not None:
                lam_pos[:, f] = gpos.detach().to("cpu", torch.float64).numpy()
            if gvel is not None:
                lam_vel[:, f] = gvel.detach().to("cpu", torch.float64).numpy()
            try:
                _, gv, gnu = h.adjoint_backward(lam_pos, lam_vel)
            finally:
                h.close()
                ctx.h = None
            dev = gpos.device if gpos is not None else gvel.device
            g_vel0 = torch.from_numpy(np.ascontiguousarray(gv[:, f])).to(dev)
            return torch.tensor(gnu, dtype=torch.float64, device=dev), g_vel0, None

    return Rollout


_ROLLOUT = None


def rollout(nu, vel0, problem: RolloutProblem):
    """Differentiable rollout: returns (pos (3, nF), vel (3, nF), alive (nF,))."""
    global _ROLLOUT
    if _ROLLOUT is None:
        _ROLLOUT = _rollout_cls()
    return _ROLLOUT.apply(nu, vel0, problem)


def dambreak_loss(pos, alive, target, x_gate: float = 0.7):
    """Squared error of the fluid centroid plus that of the mean height of the fluid beyond
    x = x_gate, against ``target`` = (cx, cy, cz, zbar). Deleted particles do not count; an
    empty gate contributes zbar = 0. Works on torch tensors and numpy arrays."""
    p = pos[:, alive]
    c = p.mean(axis=1) if isinstance(p, np.ndarray) else p.mean(dim=1)
    sel = p[0] > x_gate
    nsel = int(sel.sum())
    zbar = p[2][sel].sum() / nsel if nsel else p[2].sum() * 0.0
    t = target
    return (c[0] - t[0]) ** 2 + (c[1] - t[1]) ** 2 + (c[2] - t[2]) ** 2 + (zbar - t[3]) ** 2


def loss_target(problem: RolloutProblem, nu_target: float, vel0: np.ndarray, x_gate: float = 0.7):
    """(cx, cy, cz, zbar) of the rollout at viscosity nu_target."""
    st = problem.run(nu_target, vel0)
    f = problem.fluid
    alive = st["typ"][f] == L.FLD
    p = st["pos"][:, f][:, alive]
    sel = p[0] > x_gate
    zbar = float(p[2][sel].mean()) if sel.any() else 0.0
    return np.array([p[0].mean(), p[1].mean(), p[2].mean(), zbar])


def rollout_loss(problem: RolloutProblem, nu: float, vel0: np.ndarray, target,
                 x_gate: float = 0.7) -> float:
    """Forward-only :func:`dambreak_loss` of the rollout, summed with exact rounding
    (math.fsum), for finite-difference checks of the gradient: the loss moves by a few
    hundred ulps of a centroid coordinate for a relative viscosity step of 1e-4."""
    import math
    st = problem.run(nu, vel0)
    f = problem.fluid
    alive = st["typ"][f] == L.FLD
    p = st["pos"][:, f][:, alive]
    c = [math.fsum(p[k]) / p.shape[1] for k in range(3)]
    sel = p[0] > x_gate
    zbar = math.fsum(p[2][sel]) / int(sel.sum()) if sel.any() else 0.0
    dc = [c[k] - target[k] for k in range(3)] + [zbar - target[3]]
    return math.fsum(x * x for x in dc)
