"""Differentiable loading windows: platen reactions as a torch.autograd.Function.

A window is ``nsteps`` FP64 steps of the GPU worker with the contact topology
frozen (dem_window_forward).  Bonds may fail inside it when the device bond
hand-off is on; the failures are then fixed events of the window (the bond
state is frozen for the derivative).  Its output is the reaction of every
wall interaction group after every step, ``R[t, group, 3]`` (the values
``LsmMpi.getWallForce`` would report, Model/EWallInteractionGroup.hpp:47-53); its
differentiable inputs are the interaction parameters in the library's layout
(RotBond normalK, shearK, torsionK, bendingK per bond group; normalK, shearK per
dynamic group; the linear and rotational damping viscosities) and the initial
linear and angular velocities of every particle, rows sorted by particle id.
The backward pass is the library's hand-written reverse sweep
(dem_window_adjoint): checkpoints every ``checkpoint_every`` steps, each segment
recomputed forward on the GPU and reversed step by step.

    win = DifferentiableWindow(lsm, nsteps=2000, checkpoint_every=100)
    theta = win.parameters().requires_grad_()
    v0 = win.initial_velocities()[0].requires_grad_()
    R = win(theta, v0)                      # [nsteps, wall groups, 3]
    loss = ((R[:, :, 1] - target) ** 2).mean()
    loss.backward()                          # theta.grad, v0.grad

Calling the window again rewinds the worker to the window's start state first
(dem_window_rewind), so a calibration loop re-runs the same window with new
parameters.  Branches (touching, slipping, damping iteration counts) are those
of each forward run; the gradient is that of the branch taken.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _capi

__all__ = ["DifferentiableWindow", "PlatenWindowFunction"]


class PlatenWindowFunction(torch.autograd.Function):
    """R = window(params, vel0, angvel0); backward through dem_window_adjoint."""

    @staticmethod
    def forward(ctx, params, vel0, angvel0, window):
        R = window._run(params, vel0, angvel0)
        ctx.window = window
        ctx.generation = window._generation
        return torch.from_numpy(R)

    @staticmethod
    def backward(ctx, gR):
        w = ctx.window
        if w._generation != ctx.generation:
            raise RuntimeError("the window was run again before this backward pass")
        g = w.sim.window_adjoint(gR.detach().to(torch.float64).cpu().numpy())
        gp = torch.from_numpy(g["params"]) if ctx.needs_input_grad[0] else None
        gv = torch.from_numpy(g["vel"]) if ctx.needs_input_grad[1] else None
        gw = torch.from_numpy(g["angvel"]) if ctx.needs_input_grad[2] else None
        return gp, gv, gw, None


class DifferentiableWindow:
    """A window of ``nsteps`` steps from the worker's current state.

    ``sim`` is an ``esys.lsm.LsmMpi`` (after its set-up) or an ``_capi.DemSim``.
    """

    def __init__(self, sim, nsteps, checkpoint_every=100):
        self.sim = sim._require() if hasattr(sim, "_require") else sim
        self.nsteps = int(nsteps)
        self.checkpoint_every = int(checkpoint_every)
        self._started = False
        self._generation = 0
        p = self.sim.particles(sort=True)
        self.ids = p["id"].copy()
        self._vel0 = p["vel"].copy()
        self._angvel0 = p["angvel"].copy()

    def param_layout(self):
        return self.sim.param_layout()

    def parameters(self):
        """Current parameter vector (float64 tensor) in param_layout() order."""
        return torch.from_numpy(self.sim.param_values().copy())

    def initial_velocities(self):
        """(linear, angular) velocities at the window start, rows sorted by id."""
        return torch.from_numpy(self._vel0.copy()), torch.from_numpy(self._angvel0.copy())

    def __call__(self, params=None, vel0=None, angvel0=None):
        if params is None:
            params = self.parameters()
        return PlatenWindowFunction.apply(params, vel0, angvel0, self)

    def _run(self, params, vel0, angvel0):
        if self._started:
            self.sim.window_rewind()
        self.sim.set_params(params.detach().to(torch.float64).cpu().numpy())
        if vel0 is not None or angvel0 is not None:
            v = None if vel0 is None else np.ascontiguousarray(vel0.detach().to(torch.float64).cpu().numpy())
            w = None if angvel0 is None else np.ascontiguousarray(angvel0.detach().to(torch.float64).cpu().numpy())
            self.sim.set_particles(vel=v, angvel=w, id=self.ids.astype(np.int32))
        R = self.sim.window_forward(self.nsteps, self.checkpoint_every)
        self._started = True
        self._generation += 1
        return R
