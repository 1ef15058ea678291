"""Differentiable MLS-MPM trajectories on the B200 engine.

``Trajectory`` runs a scene (``DeviceScene`` or ``DeviceBatch``) for a fixed number of substeps from
a fixed initial state and returns the particle positions at chosen substeps, as a function of the
per-particle Lamé parameters (lambda, mu) and the initial velocity.  Its gradients come from the
engine's hand-written adjoint kernels (CrB200SolverAdjointRecord / CrB200SolverAdjointBackward:
checkpoints every ``checkpoint_interval`` substeps, recompute in between).

``trajectory(run, lam, mu, v0)`` wraps one run in a ``torch.autograd.Function`` so that losses
written in torch (and the chain rule to Young's modulus / Poisson's ratio through ``lame``) get
their gradients from the engine.  The wrapper exists for gradient checks; the engine does the work.
"""
from __future__ import annotations

import numpy as np


def lame(E, nu):
    """Lamé parameters (lambda, mu) from Young's modulus and Poisson's ratio (works on tensors)."""
    return E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), E / (2.0 * (1.0 + nu))


class Trajectory:
    """A fixed-length differentiable run of a device scene."""

    def __init__(self, ds, num_substeps: int, captures, checkpoint_interval: int = 20):
        import torch

        self.torch = torch
        self.ds = ds
        self.T = int(num_substeps)
        self.caps = [int(t) for t in captures]
        self.K = int(checkpoint_interval)
        n = self.n = ds.scene.n
        dev = ds.device
        with torch.cuda.stream(ds.stream):
            self.x0 = ds.pos[:n].clone()
            self.eye = torch.eye(3, device=dev).T.reshape(1, 9).repeat(n, 1).contiguous()  # column-major I
            self.zero9 = torch.zeros((n, 9), device=dev)
            self.out = torch.empty((len(self.caps), n, 4), device=dev)
            self.gout = torch.zeros((len(self.caps), n, 4), device=dev)
            self.gv = torch.empty((n, 4), device=dev)
            self.gm = torch.empty((n, 4), device=dev)
            self.gx = torch.empty((n, 4), device=dev)

    def forward(self, lam, mu, v0):
        """Positions (len(captures), n, 3) after the run from x0, F = I, C = 0 and velocity v0."""
        torch, ds, n = self.torch, self.ds, self.n
        ds.stream.wait_stream(torch.cuda.current_stream(ds.device))
        with torch.cuda.stream(ds.stream):
            ds.pos[:n].copy_(self.x0)
            ds.vel[:n, :3].copy_(v0.reshape(n, 3))
            ds.matp[:n, 0].copy_(lam.reshape(n))
            ds.matp[:n, 1].copy_(mu.reshape(n))
        ds.solver.set_particle_state(n, self.eye.data_ptr(), self.zero9.data_ptr(), 0)
        ds.solver.adjoint_record(self.T, self.K, self.caps, self.out.data_ptr())
        ds.sync()
        return self.out[..., :3].clone()

    def backward(self, grad_pos):
        """(dL/dlambda, dL/dmu, dL/dv0) for dL/dpositions grad_pos (len(captures), n, 3)."""
        torch, ds, n = self.torch, self.ds, self.n
        ds.stream.wait_stream(torch.cuda.current_stream(ds.device))
        with torch.cuda.stream(ds.stream):
            self.gout[..., :3].copy_(grad_pos)
        ds.solver.adjoint_backward(self.gout.data_ptr(), self.gv.data_ptr(), self.gm.data_ptr(), self.gx.data_ptr())
        ds.sync()
        return self.gm[:, 0].clone(), self.gm[:, 1].clone(), self.gv[:, :3].clone()


def _function():
    import torch

    class TrajectoryFn(torch.autograd.Function):
        @staticmethod
        def forward(ctx, lam, mu, v0, run):
            ctx.run = run
            return run.forward(lam, mu, v0)

        @staticmethod
        def backward(ctx, grad_pos):
            gl, gm, gv = ctx.run.backward(grad_pos.contiguous())
            return gl, gm, gv, None

    return TrajectoryFn


_FN = None


def trajectory(run: Trajectory, lam, mu, v0):
    """Differentiable positions at the run's captured substeps (torch.autograd.Function)."""
    global _FN
    if _FN is None:
        _FN = _function()
    return _FN.apply(lam, mu, v0, run)


def position_mse(pos, targets):
    """Sum over captured substeps of the mean squared position error (the identification loss)."""
    return ((pos - targets) ** 2).mean(dim=(1, 2)).sum()


def to_numpy(t):
    return t.detach().cpu().numpy().astype(np.float64)
