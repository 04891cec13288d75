"""Run a few time steps of one configuration: the command that ncu captures.

    python -m smectic3d_b200.profile_run --boundary neumann --precision fp32 --n 256 --steps 4

It sets a seeded U(-0.1, 0.1) field, takes ``--steps`` steps (or runs the
adjoint over ``--adjoint`` steps) and exits. The
kernel order per step is pencil (x) then plane (y,z), after one init plane and
one init pencil launch. ``ncu -k regex:plane_kernel -s 2 -c 1`` therefore
captures the plane pass of the second step.
"""
from __future__ import annotations

import argparse

import numpy as np

from .ic import noise
from .solver import Params, Solver


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--boundary", default="neumann", choices=["periodic", "neumann"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--batch", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--variant", type=int, default=0)
    ap.add_argument("--advection", action="store_true")
    ap.add_argument("--replica-block", type=int, default=0,
                    help="batched runs: replicas per L2-resident block (0 = all replicas each step)")
    ap.add_argument("--adjoint", type=int, default=0, metavar="T",
                    help="instead of plain steps, run sh_adjoint over T steps (checkpoints every 50)")
    args = ap.parse_args(argv)
    p = Params(n=args.n, batch=args.batch, boundary=args.boundary, precision=args.precision, variant=args.variant,
               advection=args.advection, replica_block=args.replica_block,
               eps_per_replica=tuple(np.linspace(-0.9, -0.5, args.batch)) if args.batch > 1 else None)
    with Solver(p) as s:
        psi = np.stack([noise(args.n, r) for r in range(args.batch)]) if args.batch > 1 else noise(args.n, 0)
        s.set_psi(psi)
        if args.adjoint:
            lam = np.zeros_like(psi)
            lam[..., 0] = 1.0
            s.adjoint(psi, args.adjoint, lam, ckpt_every=50)
        else:
            s.step(args.steps)
        s.synchronize()
    print("ok")


if __name__ == "__main__":
    main()
