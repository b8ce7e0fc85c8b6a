"""Gradients of a D(t) objective with respect to the Skyrme parameters.

The reference computes D(t) (src/hyper_vlasov.cpp:63-104 and
scripts/programs.py:82-122) but no derivatives.  This module wraps the
library's hand-written adjoint (hv_adjoint_forward / hv_adjoint_backward) as a
torch.autograd.Function, so that an objective written in torch on the D(t)
series -- such as `spectrum.power_in_band` -- can be differentiated with
respect to theta = (t0, t3, sigma, a_sym):

    run = AdjointRun(workload, particles, steps=1000, checkpoint_every=50)
    theta = torch.tensor([t0, t3, sigma, a_sym], dtype=torch.float64, requires_grad=True)
    d = dipole_series(theta, run)                     # one FP64 forward run on the GPU
    J = power_in_band(d, t, t_f, dt_row)
    J.backward()                                      # the adjoint run; theta.grad

Everything runs in FP64: on the plain path (one kernel per reference routine,
the default) or, with path=HV_PATH_FUSED, on the fused kernels (the fused
particle step, the persistent SOR for the forward and the transposed Poisson
solves).
"""
from __future__ import annotations

from dataclasses import replace

import numpy as np

from . import _lib as L
from .api import Session
from .workloads import Workload


class AdjointRun:
    """One nucleus, its initial particles and a step count; forward(theta)
    runs the FP64 forward from the initial state with checkpoints and returns
    D(t) per step, backward(dJ/dD) the gradient at that theta."""

    def __init__(self, workload: Workload, particles, steps: int, checkpoint_every: int = 50, device: int = -1,
                 path: int = L.HV_PATH_PLAIN, fast_options: dict | None = None):
        self.w = workload
        self.parts = [np.ascontiguousarray(p, dtype=np.float64) for p in particles]
        self.steps = int(steps)
        self.every = int(checkpoint_every)
        self.device = device
        self.path = int(path)
        self.fast_options = dict(fast_options or {})
        self.session = None
        self.theta = None
        self.obs = None

    def workload_at(self, theta):
        t0, t3, sigma, a_sym = (float(v) for v in theta)
        return replace(self.w, t0=t0, t3=t3, sigma=sigma, a_sym=a_sym)

    def forward(self, theta):
        self.close()
        w = self.workload_at(theta)
        self.theta = np.array([w.t0, w.t3, w.sigma, w.a_sym], dtype=np.float64)
        s = Session.from_workload(w, L.HV_F64, self.device)
        if self.fast_options:
            s.set_fast_options(**self.fast_options)
        s.upload_particles(*self.parts)
        if self.path == L.HV_PATH_PLAIN:
            s.initial_solve()  # the fused path solves the first fields with its own kernels
        self.obs = s.adjoint_forward(self.steps, self.every, self.path)
        self.session = s
        return self.obs["dipole"].copy()

    def backward(self, dJ_dD):
        if self.session is None:
            raise RuntimeError("AdjointRun.backward before forward")
        g, _ = self.session.adjoint_backward(np.asarray(dJ_dD, dtype=np.float64), self.theta)
        return g

    def objective(self, theta, fn):
        """fn(D) (numpy in, float out) of a plain forward run at theta, for
        finite differences."""
        return float(fn(self.forward(theta)))

    def close(self):
        if self.session is not None:
            self.session.close()
            self.session = None


def _function():
    import torch

    class DipoleSeries(torch.autograd.Function):
        @staticmethod
        def forward(ctx, theta, run):
            d = run.forward(theta.detach().cpu().numpy())
            ctx.run = run
            return torch.as_tensor(d, dtype=theta.dtype, device=theta.device)

        @staticmethod
        def backward(ctx, grad_d):
            g = ctx.run.backward(grad_d.detach().cpu().numpy().astype(np.float64))
            return torch.as_tensor(g, dtype=grad_d.dtype, device=grad_d.device), None

    return DipoleSeries


def dipole_series(theta, run: AdjointRun):
    """D(t) of `run` at theta (a float64 torch tensor of 4), differentiable in
    theta through the library's adjoint."""
    return _function().apply(theta, run)
