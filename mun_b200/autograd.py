"""Autograd bridges over the batched GPU solver.

``SEMLikelihoodAdjointFn`` mirrors the reference drivers' bridge
(``Bspline_Coupling/RQS_Coupling/RQS_Coupling.py:295-351``): forward returns the
log-likelihood of one control-point vector, backward multiplies the upstream gradient
by the adjoint gradient computed in the same call.

``GridLikelihood`` is the batched variant used by the flow trainer: a batch of node
values theta (B, nx*nz) of a cubic tensor B-spline grid, v = v_base + theta B^T,
returns log-likelihoods (B,) and, in backward, dL/dtheta = (dL/dv) B for every sample
(one launch sequence for the whole batch).
"""
from __future__ import annotations

import numpy as np
import torch

from .bspline import grid_basis
from .solver import Batch, SolveSpec


class SEMLikelihoodAdjointFn(torch.autograd.Function):
    """loglik(z) for control-point offsets z (2K,) around ``ctrl_pts_original``."""

    @staticmethod
    def forward(ctx, z, y_obs, noise_std, sim, ctrl_pts_original, obs_dt, obs_nt):
        if z.dim() != 1:
            raise ValueError(f"SEMLikelihoodAdjointFn expects z shape (2K,), got {tuple(z.shape)}")
        abs_ctrl = np.asarray(ctrl_pts_original, dtype=np.float64) + \
            z.detach().cpu().numpy().reshape(-1, 2)
        y = y_obs.detach().cpu().numpy() if isinstance(y_obs, torch.Tensor) else np.asarray(y_obs)
        sd = float(noise_std.detach().cpu().item()) if isinstance(noise_std, torch.Tensor) \
            else float(noise_std)
        out = sim.run_forward_and_adjoint({"bspline_ctrl": abs_ctrl, "y_obs": y, "obs_dt": float(obs_dt),
                                           "obs_nt": int(obs_nt), "noise_std": sd})
        ctx.save_for_backward(torch.as_tensor(out["grad_wrt_ctrl"], dtype=torch.float64,
                                              device=z.device))
        return torch.tensor(out["loglik"], dtype=torch.float64, device=z.device)

    @staticmethod
    def backward(ctx, grad_output):
        (g,) = ctx.saved_tensors
        return grad_output * g, None, None, None, None, None, None


class GridModel:
    """Velocity parametrisation v = v_base + theta B^T on one plan's mesh.

    The dense basis B (P, nx*nz) is held on the device; both products are plain
    GEMMs (cuBLAS)."""

    def __init__(self, plan, coords, v_base, domain, nx, nz, device="cuda"):
        self.plan = plan
        self.B = torch.as_tensor(grid_basis(np.asarray(coords), domain[0], domain[1], nx, nz),
                                 device=device)
        self.v_base = torch.as_tensor(np.asarray(v_base, dtype=np.float64), device=device)
        self.ntheta = nx * nz

    def velocity(self, theta):
        return self.v_base[None, :] + theta @ self.B.T

    def project(self, dv):
        return dv @ self.B


class GridLikelihood(torch.autograd.Function):
    """Batched log-likelihoods for theta (B, ntheta).  ``exact`` selects the exact
    discrete adjoint (sponge inside the adjoint); otherwise the reference's adjoint."""

    @staticmethod
    def forward(ctx, theta, model, y_obs, sigma, exact=True, batch=None, ckpt_k=0):
        theta = theta.detach().to(dtype=torch.float64)
        v = model.velocity(theta)
        inv_s2 = 1.0 / (float(sigma) ** 2 + 1e-24)
        n = theta.shape[0]
        specs = [SolveSpec(model.plan, v[i], adjoint=True, exact=exact, y_obs=y_obs,
                           inv_sigma2=inv_s2, ckpt_k=ckpt_k) for i in range(n)]
        (batch or Batch()).run(specs)
        st = torch.cat([s.status for s in specs])
        if bool((st != 0).any()):
            raise FloatingPointError("non-finite wavefield in the batch")
        loglik = torch.cat([s.loglik for s in specs])
        dv = torch.stack([s.grad for s in specs])          # d loglik / d v
        ctx.save_for_backward(model.project(dv))
        return loglik

    @staticmethod
    def backward(ctx, grad_output):
        (g,) = ctx.saved_tensors
        return grad_output[:, None] * g, None, None, None, None, None, None
