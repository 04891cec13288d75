"""The measurement configurations at their own sizes and lengths, shared by the
fixture generator (make_golden.py) and the GPU parity tests.

C1   periodic plain 128^3, U(-0.1, 0.1) noise (seed 0), eps = -0.75, dt = 0.05
C1'  as C1 with reference-amplitude lamellae 1.328 cos(q0 z) plus that noise
C2   Neumann 256^3, hyperboloid 0.5 cos(q0 s), R0 = 20 dx, 1e-3 U(-1, 1) noise (seed 0)
C2'  as C2 with amplitude 1.328
C3   periodic 256^3 with Stokes advection, dt = 0.02, lamellae 0.5 cos(q0 (z - 2 dx sin(2 pi x / 64 dx + phi)))
C3'  as C3 with amplitude 1.328

Long runs at 64^3 (the dominant wavenumber and the energy over 2000 steps):
L4   replica 0 of C4: periodic 64^3, eps = -0.9, U(-0.1, 0.1) noise (seed 0), dt = 0.05
L4'  periodic 64^3, eps = -0.75, 1.328 cos(q0 z) plus that noise
L2'  Neumann 64^3, eps = -0.75, hyperboloid of amplitude 1.328, R0 = 12 dx (seed 0)

The reference's own size, 512^3 (two steps; FP64 and FP32):
X2   Neumann 512^3, hyperboloid of amplitude 1.328, R0 = 40 dx (seed 0)
X1   periodic 512^3, 1.328 cos(q0 z) plus U(-0.1, 0.1) noise (seed 0)

beta = 2, gamma = 1, alpha = q0 = 1, dx = 2 pi / 8 throughout; eps = -0.75 unless stated.  A case records
the states after ``checks`` steps, subsampled every ``stride`` points per axis,
with global sums, the energy and the dominant wavenumber; the advected cases
also record the surfTrack pass (one more step) on every ``surf_stride``-th column.
"""
from __future__ import annotations

import math

import numpy as np

from smectic3d_b200 import ic

DX = 2.0 * math.pi / 8.0

CASES = {
    "c1_periodic128": dict(boundary="periodic", n=128, dt=0.05, ic="noise", amp=None, checks=(100, 500), stride=4),
    "c1p_periodic128_amp1328": dict(boundary="periodic", n=128, dt=0.05, ic="lamellae+noise", amp=1.328,
                                    checks=(100, 500), stride=4),
    "c2_neumann256": dict(boundary="neumann", n=256, dt=0.05, ic="hyperboloid", amp=0.5, checks=(100,), stride=8),
    "c2p_neumann256_amp1328": dict(boundary="neumann", n=256, dt=0.05, ic="hyperboloid", amp=1.328, checks=(100,),
                                   stride=8),
    "c3_advected256": dict(boundary="periodic", n=256, dt=0.02, ic="undulated", amp=0.5, checks=(20,), stride=8,
                           advect=True, surf_stride=4),
    "c3p_advected256_amp1328": dict(boundary="periodic", n=256, dt=0.02, ic="undulated", amp=1.328, checks=(20,),
                                    stride=8, advect=True, surf_stride=4),
    "l4_periodic64_eps09": dict(boundary="periodic", n=64, dt=0.05, eps=-0.9, ic="noise", amp=None,
                                checks=(500, 1000, 2000), stride=4),
    "l4p_periodic64_amp1328": dict(boundary="periodic", n=64, dt=0.05, ic="lamellae+noise", amp=1.328,
                                   checks=(500, 1000, 2000), stride=4),
    "l2p_neumann64_amp1328": dict(boundary="neumann", n=64, dt=0.05, ic="hyperboloid", amp=1.328, r0_cells=12.0,
                                  checks=(500, 1000, 2000), stride=4),
    "x2_neumann512": dict(boundary="neumann", n=512, dt=0.05, ic="hyperboloid", amp=1.328, r0_cells=40.0,
                          checks=(2,), stride=16),
    "x1_periodic512": dict(boundary="periodic", n=512, dt=0.05, ic="lamellae+noise", amp=1.328, checks=(2,),
                           stride=16),
}


def initial_condition(cfg: dict) -> np.ndarray:
    n = cfg["n"]
    kind = cfg["ic"]
    if kind == "noise":
        return ic.noise(n, 0)
    if kind == "lamellae+noise":
        return cfg["amp"] * np.cos(np.arange(n) * DX)[None, None, :] + ic.noise(n, 0)
    if kind == "hyperboloid":
        return ic.hyperboloid(n, DX, amp=cfg["amp"], r0_cells=cfg.get("r0_cells", 20.0), seed=0)
    if kind == "undulated":
        return ic.undulated_lamellae(n, DX, amp=cfg["amp"], seed=0)
    raise ValueError(kind)


def subsample(psi: np.ndarray, stride: int) -> np.ndarray:
    return psi[::stride, ::stride, ::stride].copy()
