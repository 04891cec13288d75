"""PyTorch autograd over the time loop, backed by the discrete adjoint.

``sh_evolve(psi0, eps, q0, params, nsteps)`` runs ``nsteps`` CNAB2 steps of the
periodic plain step (the configuration ``sh_adjoint`` differentiates) and
returns psi^T; its backward pass calls ``sh_adjoint`` with the incoming
gradient of psi^T and returns dL/dpsi0, dL/deps and dL/dq0 (FP64 sums, one
checkpoint every ``ckpt_every`` steps).  The forward and the backward run in
the handle's precision; tensors cross as float64 on the host.

    psiT = sh_evolve(psi0, eps, q0, Params(n=128, precision="fp32"), 1000)
    loss = 0.5 * ((psiT - target) ** 2).sum()
    loss.backward()          # psi0.grad, eps.grad, q0.grad
"""
from __future__ import annotations

import dataclasses

import numpy as np
import torch

from .solver import Params, Solver


class _Evolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, psi0, eps, q0, params, nsteps, ckpt_every):
        p = dataclasses.replace(params, eps=float(eps), q0=float(q0), batch=1)
        psi0_np = psi0.detach().to("cpu", torch.float64).numpy()
        with Solver(p) as s:
            s.set_psi(psi0_np)
            s.step(int(nsteps))
            psiT = s.get_psi()
        ctx.p, ctx.nsteps, ctx.ckpt_every = p, int(nsteps), int(ckpt_every)
        ctx.scalar_like = ((eps.dtype, eps.device), (q0.dtype, q0.device))
        ctx.save_for_backward(psi0)
        return torch.as_tensor(psiT, device=psi0.device)

    @staticmethod
    def backward(ctx, grad_psiT):
        (psi0,) = ctx.saved_tensors
        g = grad_psiT.detach().to("cpu", torch.float64).numpy()
        with Solver(ctx.p) as s:
            ge, gq, gp = s.adjoint(psi0.detach().to("cpu", torch.float64).numpy(), ctx.nsteps, g, ctx.ckpt_every)
        (edt, edev), (qdt, qdev) = ctx.scalar_like
        return (torch.as_tensor(gp, device=psi0.device).to(psi0.dtype),
                torch.tensor(float(ge[0]), dtype=edt, device=edev),
                torch.tensor(float(gq[0]), dtype=qdt, device=qdev), None, None, None)


def sh_evolve(psi0: torch.Tensor, eps, q0, params: Params, nsteps: int, ckpt_every: int = 50) -> torch.Tensor:
    """psi^T after ``nsteps`` steps from ``psi0``, differentiable in psi0, eps and q0."""
    eps = eps if torch.is_tensor(eps) else torch.tensor(float(eps), dtype=torch.float64)
    q0 = q0 if torch.is_tensor(q0) else torch.tensor(float(q0), dtype=torch.float64)
    return _Evolve.apply(psi0, eps, q0, params, nsteps, ckpt_every)
