"""Initial conditions: the reference's analytic ICs and the seeded synthetic ICs
of the benchmark workloads.  All return float64 arrays indexed (i, j, k) with
k (z) fastest, grid spacing ``dx`` in every direction.
"""
from __future__ import annotations

import math

import numpy as np


def _idx(n):
    return np.arange(n, dtype=np.float64)


def noise(n: int, seed: int, amp: float = 0.1) -> np.ndarray:
    """i.i.d. U(-amp, amp) from numpy.random.default_rng(seed)."""
    return np.random.default_rng(seed).uniform(-amp, amp, size=(n, n, n))


def noise_batch(n: int, seeds, amp: float = 0.1) -> np.ndarray:
    return np.stack([noise(n, s, amp) for s in seeds])


def hyperboloid(n: int, dx: float, q0: float = 1.0, amp: float = 0.5, r0_cells: float = 20.0,
                noise_amp: float = 1e-3, seed: int = 0) -> np.ndarray:
    """psi0 = amp cos(q0 s), s = sqrt(max(x^2 + y^2 - z^2 + R0^2, 0)), centred in
    the box, R0 = r0_cells dx, plus noise_amp U(-1, 1)."""
    c = (_idx(n) - n / 2) * dx
    x, y, z = c[:, None, None], c[None, :, None], c[None, None, :]
    r0 = r0_cells * dx
    s = np.sqrt(np.maximum(x * x + y * y - z * z + r0 * r0, 0.0))
    psi = amp * np.cos(q0 * s)
    if noise_amp:
        psi = psi + noise_amp * np.random.default_rng(seed).uniform(-1.0, 1.0, size=(n, n, n))
    return psi


def undulated_lamellae(n: int, dx: float, q0: float = 1.0, amp: float = 0.5, und_cells: float = 2.0,
                       wavelength_cells: float = 64.0, seed: int = 0) -> np.ndarray:
    """psi = amp cos(q0 (z - A sin(2 pi x / lambda + phi))), A = und_cells dx,
    lambda = wavelength_cells dx, phi drawn from default_rng(seed)."""
    phi = np.random.default_rng(seed).uniform(0.0, 2.0 * math.pi)
    x = _idx(n)[:, None, None] * dx
    z = _idx(n)[None, None, :] * dx
    h = und_cells * dx * np.sin(2.0 * math.pi * x / (wavelength_cells * dx) + phi)
    return np.broadcast_to(amp * np.cos(q0 * (z - h)), (n, n, n)).copy()


def pf3d_lamellae(n: int, dx: float, q0: float = 1.0, amp: float = 1.2441, qi: float = 0.5,
                  kmin: int | None = None, kmax: int | None = None) -> np.ndarray:
    """periodicFFT/pf3d.cpp:302-324: Amp cos(q0 k dz) + 0.1 Amp sin(q0 k dz)
    (cos(Qi i dx) + cos(Qi j dy)) for kmin < k < kmax (24 and 232 at N = 256), else 0."""
    if kmin is None:
        kmin = int(round(24 * n / 256))
    if kmax is None:
        kmax = int(round(232 * n / 256))
    i = _idx(n)[:, None, None]
    j = _idx(n)[None, :, None]
    k = _idx(n)[None, None, :]
    psi = amp * np.cos(q0 * k * dx) + amp * 0.1 * np.sin(q0 * k * dx) * (np.cos(qi * i * dx) + np.cos(qi * j * dx))
    mask = (k > kmin) & (k < kmax)
    return np.where(mask, psi, 0.0)


def pf3dval_mode(n: int, dx: float, mqz: float, amp: float = 1e-4) -> np.ndarray:
    """periodicFFT/pf3dVal.cpp:219-229: 1e-4 cos(mqZ k dz)."""
    k = _idx(n)[None, None, :]
    return np.broadcast_to(amp * np.cos(mqz * k * dx), (n, n, n)).copy()


def _ellipse_profile(n, dx, q0, amp, a_e, b_e, zs, ds, mid):
    """Shared ellipse/torus morphology of cosNoAdvMorph and pf3dMorph."""
    inside = np.sqrt(((ds - mid) / a_e) ** 2 + (zs / b_e) ** 2) <= 1.0
    tor = amp * np.cos(q0 * dx * np.sqrt(((b_e / a_e) * (ds - mid)) ** 2 + zs * zs))
    flat = np.where(np.abs(zs) < b_e, amp * np.cos(q0 * zs * dx), 0.0)
    return np.where(ds < mid, np.where(inside, tor, 0.0), flat)


def cos_bottom_hyperboloid(n: int, dx: float, q0: float = 1.0, amp: float = 1.328, a_e: float | None = None,
                           b_e: float | None = None) -> np.ndarray:
    """cosFFT/mesabi/cosNoAdvMorph.cpp:289-331 (aE=312, bE=376 at N=512),
    focal-conic profile resting on the k = 0 wall."""
    a_e = 312.0 * n / 512 if a_e is None else a_e
    b_e = 376.0 * n / 512 if b_e is None else b_e
    mid = n / 2
    i = _idx(n)[:, None, None]
    j = _idx(n)[None, :, None]
    k = _idx(n)[None, None, :]
    xs, ys, zs = i - mid, j - mid, k + 0.0 * i
    ds = np.sqrt(xs * xs + ys * ys) + 0.0 * k
    psi = _ellipse_profile(n, dx, q0, amp, a_e, b_e, zs, ds, mid)
    return np.where(k < b_e + 1, psi, 0.0)


def pf3dmorph_torus(n: int, dx: float, q0: float = 1.0, amp: float = 1.328, a_e: float | None = None,
                    b_e: float | None = None) -> np.ndarray:
    """periodicFFT/pf3dMorph.cpp:331-376 (aE=245, bE=180, 62 < k < 450 at N=512),
    centred in z."""
    a_e = 245.0 * n / 512 if a_e is None else a_e
    b_e = 180.0 * n / 512 if b_e is None else b_e
    kmin, kmax = 62 * n / 512, 450 * n / 512
    mid = n / 2
    i = _idx(n)[:, None, None]
    j = _idx(n)[None, :, None]
    k = _idx(n)[None, None, :]
    xs, ys, zs = i - mid, j - mid, (k - mid) + 0.0 * i
    ds = np.sqrt(xs * xs + ys * ys) + 0.0 * k
    psi = _ellipse_profile(n, dx, q0, amp, a_e, b_e, zs, ds, mid)
    return np.where((k > kmin) & (k < kmax), psi, 0.0)
