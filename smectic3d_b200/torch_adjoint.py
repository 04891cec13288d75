"""PyTorch autograd over the time loop, backed by the discrete adjoint.

``sh_evolve(psi0, eps, q0, params, nsteps)`` runs ``nsteps`` CNAB2 steps of the
periodic plain step (the configuration ``sh_adjoint`` differentiates) and
returns psi^T.  The forward pass is ``sh_adjoint_forward``: the time loop
keeping one checkpoint every ``ckpt_every`` steps on the device.  The backward
pass is ``sh_adjoint_backward`` on the same handle: it recomputes each segment
from those checkpoints and runs the reverse sweep for the incoming gradient of
psi^T, returning dL/dpsi0, dL/deps and dL/dq0 (FP64 sums).  The forward is not
run a second time.  Both run in the handle's precision; tensors cross as
float64 on the host.  The handle (and its checkpoints) lives until the
backward pass has run or the graph is freed.

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
        s = Solver(p)
        try:
            s.adjoint_forward(psi0_np, int(nsteps), int(ckpt_every))
            psiT = s.get_psi()
        except BaseException:
            s.close()
            raise
        ctx.solver = s
        ctx.scalar_like = ((eps.dtype, eps.device), (q0.dtype, q0.device))
        ctx.psi_like = (psi0.dtype, psi0.device)
        return torch.as_tensor(psiT, device=psi0.device)

    @staticmethod
    def backward(ctx, grad_psiT):
        g = grad_psiT.detach().to("cpu", torch.float64).numpy()
        s = ctx.solver
        try:
            ge, gq, gp = s.adjoint_backward(g)
        finally:
            s.close()
            ctx.solver = None
        (edt, edev), (qdt, qdev) = ctx.scalar_like
        pdt, pdev = ctx.psi_like
        return (torch.as_tensor(gp, device=pdev).to(pdt),
                torch.tensor(float(ge[0]), dtype=edt, device=edev),
                torch.tensor(float(gq[0]), dtype=qdt, device=qdev), None, None, None)


def sh_evolve(psi0: torch.Tensor, eps, q0, params: Params, nsteps: int, ckpt_every: int = 50) -> torch.Tensor:
    """psi^T after ``nsteps`` steps from ``psi0``, differentiable in psi0, eps and q0."""
    eps = eps if torch.is_tensor(eps) else torch.tensor(float(eps), dtype=torch.float64)
    q0 = q0 if torch.is_tensor(q0) else torch.tensor(float(q0), dtype=torch.float64)
    return _Evolve.apply(psi0, eps, q0, params, nsteps, ckpt_every)
