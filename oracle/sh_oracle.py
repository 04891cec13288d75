"""FP64 CPU oracle for the smectic3D per-step Swift-Hohenberg update.

TEST INFRASTRUCTURE ONLY.  This module is the checker that the CUDA path is
compared against; it is imported by ``tests/``, by ``__graft_entry__.smoke()``
and by the CPU-baseline leg of ``bench.py`` and by nothing else.  The product
path never calls it.

It is a line-by-line restatement of the reference's time loops in NumPy/SciPy
(pocketfft, double precision) in place of FFTW 3.3-MPI, which the reference
links and which is not available here:

* periodic plain step           periodicFFT/pf3dVal.cpp:247-301
* periodic advected step        periodicFFT/pf3d.cpp:162-222, 363-485
* pinning penalty (option)      periodicFFT/pf3dMorph.cpp:456-467, 572-589
* surfTrack surface pass        periodicFFT/surfTrack.cpp:602-626, 767-806
* Neumann (DCT) step            cosFFT/mesabi/cosNoAdvMorph.cpp:112, 216-231,
                                423-442, 483-530
* substrate penalty (option)    cosFFT/comet/cosNoAdvMorph.cpp:67-74, 480-540,
                                591-623
* L1 monitor                    periodicFFT/pf3d.cpp:489-518
* energy functional             energyPsi.m:217-234 (FD + trapz form) and its
                                spectral restatement

Parity status: UNPINNED against the reference's own outputs.  The reference
has no tests, golden files or fixtures and cannot be compiled here (it needs
fftw3-mpi and an MPI C++ compiler), so no reference output exists to pin
against.  The oracle is instead pinned to analytic known-answer tests
(tests/test_oracle.py): transform scale conventions of FFTW's R2C/C2R and
REDFT10/REDFT01, the exact CNAB2 growth factor of grid modes, the lamellar
amplitude and Lyapunov decrease, the Stokes projector identities and the
surfTrack crossing of a planar front.

Conventions kept from the reference:
* SciPy ``rfftn``/``irfftn`` equal FFTW's unnormalised r2c/c2r, including the
  c2r treatment of non-Hermitian data on the kz=0 and kz=N/2 planes (complex
  inverse over x and y, then the real part of those planes).
* ``dctn(type=2)`` / ``dctn(type=3)`` with norm=None equal REDFT10 / REDFT01.
* The Nyquist wavenumber is +pi/dx (periodicFFT/pf3d.cpp:166-190).
* The first step uses N^{-1} := N(psi^0) without advection (Euler start,
  periodicFFT/pf3d.cpp:363-374).
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np
import scipy.fft as sfft

WORKERS = os.cpu_count() or 1


@dataclasses.dataclass
class Params:
    """Runtime copy of the constants the reference hard-codes in main().

    periodicFFT/pf3d.cpp:46-73, cosFFT/mesabi/cosNoAdvMorph.cpp:89-112.
    """
    n: int = 32
    dx: float = 2.0 * np.pi / 8.0
    dt: float = 0.05
    eps: float = -0.75
    beta: float = 2.0
    gamma: float = 1.0
    alpha: float = 1.0
    q0: float = 1.0
    eta: float = 1.0
    rho: float = 1.0
    nonlinearity: str = "quintic"   # "quintic": b psi^3 - g psi^5 ; "quad_cubic": b psi^2 - g psi^3
    scheme: str = "cnab2"           # "cnab2" (reference) or "imex_euler"
    w_mid: float = 0.0              # pinning penalty weight (pf3dMorph wMid)
    sub_sigma: float = 0.0          # substrate penalty sigma (comet cosNoAdvMorph)
    sub_z0: float = 1e-4


# ---------------------------------------------------------------------------
# wavenumbers
# ---------------------------------------------------------------------------

def kvec_periodic(n: int, dx: float) -> np.ndarray:
    """Vq[i] = 2 pi i/(dx N) for i <= N/2, else -(N-i) 2 pi/(dx N).

    periodicFFT/pf3d.cpp:162-190: the Nyquist entry is +pi/dx.
    """
    q = np.empty(n)
    for i in range(n):
        if i < n // 2 + 1:
            q[i] = 2.0 * np.pi * i / (dx * n)
        else:
            q[i] = -(n - i) * 2.0 * np.pi / (dx * n)
    return q


def kvec_dct(n: int, dx: float) -> np.ndarray:
    """Vq[m] = pi m/(dx N), cosFFT/mesabi/cosNoAdvMorph.cpp:216-231."""
    return np.pi * np.arange(n) / (dx * n)


def _grids_periodic(p: Params):
    q = kvec_periodic(p.n, p.dx)
    qx = q[:, None, None]
    qy = q[None, :, None]
    qz = q[None, None, : p.n // 2 + 1]
    return qx, qy, qz


def _grids_dct(p: Params):
    q = kvec_dct(p.n, p.dx)
    return q[:, None, None], q[None, :, None], q[None, None, :]


def _tables(mq2, p: Params):
    """opSH, aLin, C1, C2 (periodicFFT/pf3d.cpp:195-216)."""
    op_sh = p.alpha * (mq2 - p.q0 * p.q0) ** 2
    a_lin = p.eps - op_sh
    c1 = 1.0 + 0.5 * p.dt * a_lin
    c2 = 1.0 - 0.5 * p.dt * a_lin
    return op_sh, a_lin, c1, c2


# ---------------------------------------------------------------------------
# nonlinearity
# ---------------------------------------------------------------------------

def nonlin(psi: np.ndarray, p: Params) -> np.ndarray:
    """N(psi) = beta psi^3 - gamma psi^5 (periodicFFT/pf3d.cpp:368-369).

    ``quad_cubic`` selects beta psi^2 - gamma psi^3 instead.
    """
    if p.nonlinearity == "quintic":
        return p.beta * psi ** 3 - p.gamma * psi ** 5
    if p.nonlinearity == "quad_cubic":
        return p.beta * psi ** 2 - p.gamma * psi ** 3
    raise ValueError(p.nonlinearity)


def nonlin_deriv(psi: np.ndarray, p: Params) -> np.ndarray:
    if p.nonlinearity == "quintic":
        return 3.0 * p.beta * psi ** 2 - 5.0 * p.gamma * psi ** 4
    return 2.0 * p.beta * psi - 3.0 * p.gamma * psi ** 2


def pin_penalty(psi: np.ndarray, p: Params, dz: float) -> np.ndarray:
    """2 wMid (psi[k-1] - 2 psi[k] + psi[k+1]) / dz^2 on the plane k = Nz/2.

    periodicFFT/pf3dMorph.cpp:456-467.
    """
    out = np.zeros_like(psi)
    if p.w_mid != 0.0:
        m = psi.shape[2] // 2
        out[:, :, m] = 2.0 * p.w_mid * (psi[:, :, m - 1] - 2.0 * psi[:, :, m] + psi[:, :, m + 1]) / (dz * dz)
    return out


# ---------------------------------------------------------------------------
# periodic solver (R2C / C2R)
# ---------------------------------------------------------------------------

def r2c(a):
    return sfft.rfftn(a, workers=WORKERS)


def c2r(a, n):
    """Unnormalised inverse (FFTW c2r convention)."""
    return sfft.irfftn(a, s=(n, n, n), norm="forward", workers=WORKERS)


class PeriodicOracle:
    """Periodic SH integrator (plain or with Stokes advection).

    State: psi (real, dense (N,N,N)) and NqPast (half spectrum).
    """

    def __init__(self, psi0: np.ndarray, p: Params, advect: bool = False):
        self.p = p
        self.n = p.n
        self.advect = advect
        self.scale = 1.0 / float(self.n) ** 3
        qx, qy, qz = _grids_periodic(p)
        self.qx, self.qy, self.qz = qx, qy, qz
        self.mq2 = qx * qx + qy * qy + qz * qz
        self.op_sh, self.a_lin, self.c1, self.c2 = _tables(self.mq2, p)
        with np.errstate(divide="ignore", invalid="ignore"):
            cm1 = 1.0 / (p.rho * p.eta * self.mq2)
            cm2x = qx / self.mq2
            cm2y = qy / self.mq2
            cm2z = qz / self.mq2
        # periodicFFT/pf3d.cpp:219-222: zero mode of the Stokes tables
        cm1[0, 0, 0] = 0.0
        cm2x = np.broadcast_to(cm2x, self.mq2.shape).copy()
        cm2y = np.broadcast_to(cm2y, self.mq2.shape).copy()
        cm2z = np.broadcast_to(cm2z, self.mq2.shape).copy()
        cm2x[0, 0, 0] = cm2y[0, 0, 0] = cm2z[0, 0, 0] = 0.0
        self.cm1, self.cm2x, self.cm2y, self.cm2z = cm1, cm2x, cm2y, cm2z
        self.psi = np.array(psi0, dtype=np.float64, copy=True)
        self.dz = p.dx
        # First NqPast, discarding advection (periodicFFT/pf3d.cpp:363-374)
        self.nq_past = r2c(self._nonlin_local(self.psi))
        self.step_count = 0
        self.last = {}

    def _nonlin_local(self, psi):
        return nonlin(psi, self.p) + pin_penalty(psi, self.p, self.dz)

    def velocity(self, psiq):
        """Stokes velocity from S = (L psi) grad psi.

        periodicFFT/pf3d.cpp:399-451.  Returns (u, grad, lpsi).
        """
        n, s = self.n, self.scale
        gx = c2r(s * 1j * self.qx * psiq, n)
        gy = c2r(s * 1j * self.qy * psiq, n)
        gz = c2r(s * 1j * self.qz * psiq, n)
        lpsi = c2r(s * self.op_sh * psiq, n)
        sqx = r2c(lpsi * gx)
        sqy = r2c(lpsi * gy)
        sqz = r2c(lpsi * gz)
        dot = self.qx * sqx + self.qy * sqy + self.qz * sqz
        ux = c2r(s * self.cm1 * (sqx - self.cm2x * dot), n)
        uy = c2r(s * self.cm1 * (sqy - self.cm2y * dot), n)
        uz = c2r(s * self.cm1 * (sqz - self.cm2z * dot), n)
        return (ux, uy, uz), (gx, gy, gz), lpsi

    def step(self):
        """One time step (periodicFFT/pf3d.cpp:395-485; pf3dVal.cpp:276-301)."""
        p, n, s = self.p, self.n, self.scale
        psi = self.psi
        psiq = r2c(psi)
        nr = self._nonlin_local(psi)
        grads = None
        if self.advect:
            (ux, uy, uz), grads, _ = self.velocity(psiq)
            nr = nr - ux * grads[0] - uy * grads[1] - uz * grads[2]
        nq = r2c(nr)
        if p.scheme == "cnab2":
            psiq_new = s * (self.c1 * psiq + 0.5 * p.dt * (3.0 * nq - self.nq_past)) / self.c2
        elif p.scheme == "imex_euler":
            psiq_new = s * (psiq + p.dt * nq) / (1.0 - p.dt * self.a_lin)
        else:
            raise ValueError(p.scheme)
        psi_new = c2r(psiq_new, n)
        self.last = {"psiq": psiq, "nq": nq, "grads": grads, "psi_old": psi}
        self.nq_past = nq
        self.psi = psi_new
        self.step_count += 1
        return psi_new

    def run(self, steps: int):
        for _ in range(steps):
            self.step()
        return self.psi

    # -- surfTrack --------------------------------------------------------
    def surface_fields(self):
        """Spectral fields surfTrack builds in its step.

        periodicFFT/surfTrack.cpp:602-626, using the values of the step just
        taken (psi^n spectrum, N^n).  The reference builds the curvature
        spectra from arrays it has already passed to FFTW c2r plans, which
        FFTW may overwrite; this restates the intended -q_a q_b psiq form.
        """
        n, s = self.n, self.scale
        psiq, nq = self.last["psiq"], self.last["nq"]
        grads = self.last["grads"]
        if grads is None:
            grads = (c2r(s * 1j * self.qx * psiq, n), c2r(s * 1j * self.qy * psiq, n),
                     c2r(s * 1j * self.qz * psiq, n))
        dtpsi = c2r(s * (self.a_lin * psiq + nq), n)
        dxx = c2r(-s * self.qx * self.qx * psiq, n)
        dyy = c2r(-s * self.qy * self.qy * psiq, n)
        dxy = c2r(-s * self.qx * self.qy * psiq, n)
        curvh = c2r(-s * (self.qx * self.qx + self.qy * self.qy) * psiq, n)
        return grads, dtpsi, curvh, dxx, dyy, dxy


def surface_scan_vec(psi_new, grads, dtpsi, curvh, dxx, dyy, dxy, threshold: float = 0.1):
    """``surface_scan`` written with whole-array operations, for grids where
    the per-column loop is too slow (equal to it, tests/test_oracle.py)."""
    n = psi_new.shape[0]
    k = np.arange(n)[None, None, :]
    above = psi_new > threshold
    has1 = above.any(axis=2)
    k1 = np.argmax(above, axis=2)
    neg = (psi_new < 0) & (k > k1[:, :, None])
    found = has1 & neg.any(axis=2)
    k2 = np.argmax(neg, axis=2)
    ii, jj = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    km = np.maximum(k2 - 1, 0)
    back = np.abs(psi_new[ii, jj, k2]) > np.abs(psi_new[ii, jj, km])
    idx = np.where(back, km, k2)
    pick = lambda f: f[ii, jj, idx]
    gv = np.sqrt(pick(grads[0]) ** 2 + pick(grads[1]) ** 2 + pick(grads[2]) ** 2)
    z = np.where(found, k2, -1).astype(np.int64)
    with np.errstate(divide="ignore", invalid="ignore"):
        vn = np.where(found, pick(dtpsi) / gv, np.nan)
        hh = np.where(found, pick(curvh) / gv, np.nan)
        kk = np.where(found, (pick(dxx) * pick(dyy) - pick(dxy) ** 2) / (gv * gv), np.nan)
    return z, vn, hh, kk


def surface_scan(psi_new, grads, dtpsi, curvh, dxx, dyy, dxy, threshold: float = 0.1):
    """Column scan of surfTrack (periodicFFT/surfTrack.cpp:767-806).

    For each (i, j) scan +z for the first psi < 0 after psi > threshold;
    step back one voxel if that one is closer to zero.  Returns z (the
    reference writes the unadjusted k), v_n, H, K per column, NaN / -1 where
    no crossing exists.
    """
    n = psi_new.shape[0]
    z = -np.ones((n, n), dtype=np.int64)
    vn = np.full((n, n), np.nan)
    hh = np.full((n, n), np.nan)
    kk = np.full((n, n), np.nan)
    for i in range(n):
        for j in range(n):
            col = psi_new[i, j]
            track = 0
            for k in range(n):
                if col[k] > threshold and track == 0:
                    track = 1
                if col[k] < 0 and track == 1:
                    idx = k
                    if abs(col[k]) > abs(col[k - 1]):
                        idx = k - 1
                    z[i, j] = k
                    gv = np.sqrt(grads[0][i, j, idx] ** 2 + grads[1][i, j, idx] ** 2 + grads[2][i, j, idx] ** 2)
                    vn[i, j] = dtpsi[i, j, idx] / gv
                    hh[i, j] = curvh[i, j, idx] / gv
                    kk[i, j] = (dxx[i, j, idx] * dyy[i, j, idx] - dxy[i, j, idx] ** 2) / (gv * gv)
                    track = 2
                    break
    return z, vn, hh, kk


# ---------------------------------------------------------------------------
# Neumann solver (REDFT10 / REDFT01)
# ---------------------------------------------------------------------------

def dct3d(a):
    return sfft.dctn(a, type=2, workers=WORKERS)


def idct3d(a):
    return sfft.dctn(a, type=3, workers=WORKERS)


def kvec_dst(n: int, dx: float) -> np.ndarray:
    """Vs[m] = pi (m + 1)/(dx N), the RODFT10 wavenumbers (cosFFT/comet/morphSurfK.cpp:331-348)."""
    return np.pi * (np.arange(n) + 1.0) / (dx * n)


def dst3d(a):
    """RODFT10 in every axis (FFTW's unnormalised DST-II)."""
    return sfft.dstn(a, type=2, workers=WORKERS)


def idst3d(a):
    """RODFT01 in every axis (FFTW's unnormalised DST-III)."""
    return sfft.dstn(a, type=3, workers=WORKERS)


class NeumannOracle:
    """cosNoAdvMorph: DCT-II forward, DCT-III inverse, scale 0.125/N^3.

    cosFFT/mesabi/cosNoAdvMorph.cpp:112, 216-231, 423-442, 483-530.
    Substrate penalty: cosFFT/comet/cosNoAdvMorph.cpp:67-74, 591-623.
    advect=True: the Stokes velocity of cosFFT/comet/morphSurfK.cpp (sine
    transforms, :331-348, 390-418, 686-770, 862-882) advects psi as the
    periodic step does, N = beta psi^3 - gamma psi^5 - u . grad psi (the term
    morphSurfK.cpp:893-898 carries commented out); the first history N-hat
    has no advection, as in morphSurfK.cpp:629-636.
    """

    def __init__(self, psi0: np.ndarray, p: Params, advect: bool = False):
        self.p = p
        self.n = p.n
        self.advect = advect
        self.scale = 0.125 / float(self.n) ** 3
        qx, qy, qz = _grids_dct(p)
        self.qx, self.qy, self.qz = qx, qy, qz
        self.mq2 = qx * qx + qy * qy + qz * qz
        self.op_sh, self.a_lin, self.c1, self.c2 = _tables(self.mq2, p)
        self.substrate = -self.scale * (qx * qx + qy * qy)
        k = np.arange(self.n, dtype=np.float64)
        # wallPotential(k) = sigma exp(-k/z0) (comet cosNoAdvMorph.cpp:67-74)
        with np.errstate(over="ignore", under="ignore"):
            self.wall = (p.sub_sigma * np.exp(-k / p.sub_z0))[None, None, :]
        self.psi = np.array(psi0, dtype=np.float64, copy=True)
        self.dz = p.dx
        self.nq = dct3d(self._nonlin_local(self.psi))
        self.step_count = 0
        self.last = {}

    def _nonlin_local(self, psi):
        out = nonlin(psi, self.p) + pin_penalty(psi, self.p, self.dz)
        if self.p.sub_sigma != 0.0:
            pen = idct3d(self.substrate * dct3d(psi))
            out = out + pen * self.wall
        return out

    def velocity(self, psiq):
        """Stokes velocity of the Neumann box (cosFFT/comet/morphSurfK.cpp):
        L psi = REDFT01(scale opSH psihat) (:686-696); grad psi by centred
        differences, one-sided at the walls (:700-766); S = (L psi) grad psi
        through RODFT10 (:763-770); u = RODFT01(CM1 (S - CM2 (Vs . S))) with the
        sine wavenumbers Vs = pi (m+1)/L in every axis, CM1 = scale/(rho eta |Vs|^2),
        CM2 = Vs/|Vs|^2 (:624-631, 862-882).  Returns (u, grad, L psi)."""
        p, s = self.p, self.scale
        psi = self.psi
        lpsi = idct3d(s * self.op_sh * psiq)
        grads = tuple(_fd_wall(psi, ax, p.dx) for ax in range(3))
        vs = kvec_dst(self.n, p.dx)
        vx, vy, vz = vs[:, None, None], vs[None, :, None], vs[None, None, :]
        mq2 = vx * vx + vy * vy + vz * vz
        cm1 = s / (p.rho * p.eta * mq2)
        sq = [dst3d(lpsi * g) for g in grads]
        dot = vx * sq[0] + vy * sq[1] + vz * sq[2]
        u = tuple(idst3d(cm1 * (sc - vc / mq2 * dot)) for sc, vc in zip(sq, (vx, vy, vz)))
        return u, grads, lpsi

    def step(self):
        p = self.p
        nq_past = self.nq
        nr = self._nonlin_local(self.psi)
        psiq = dct3d(self.psi)
        grads = u = None
        if self.advect:
            u, grads, _ = self.velocity(psiq)
            nr = nr - u[0] * grads[0] - u[1] * grads[1] - u[2] * grads[2]
        nq = dct3d(nr)
        if p.scheme == "cnab2":
            psiq_new = self.scale * (self.c1 * psiq + 0.5 * p.dt * (3.0 * nq - nq_past)) / self.c2
        else:
            psiq_new = self.scale * (psiq + p.dt * nq) / (1.0 - p.dt * self.a_lin)
        psi_new = idct3d(psiq_new)
        self.last = {"psiq": psiq, "nq": nq, "psi_old": self.psi, "u": u, "grads": grads}
        self.nq = nq
        self.psi = psi_new
        self.step_count += 1
        return psi_new

    def run(self, steps: int):
        for _ in range(steps):
            self.step()
        return self.psi


def _fd_wall(a, axis, h):
    """Centred difference along ``axis`` with the one-sided walls of the
    Neumann curvature pass: (a[i+1] - a[i-1]) / 2h inside, 2 (a[1] - a[0]) / 2h
    and 2 (a[-1] - a[-2]) / 2h at the walls (cosNoAdvMorphCurv.cpp:811-872)."""
    a = np.moveaxis(a, axis, 0)
    g = np.empty_like(a)
    g[1:-1] = (a[2:] - a[:-2]) / (2 * h)
    g[0] = 2 * (a[1] - a[0]) / (2 * h)
    g[-1] = 2 * (a[-1] - a[-2]) / (2 * h)
    return np.moveaxis(g, 0, axis)


def neumann_curvature_fields(orc: "NeumannOracle"):
    """Spectral fields of the curvature pass at the oracle's current psi
    (cosFFT/comet/cosNoAdvMorphCurv.cpp:742-770): psi_xx, psi_yy, psi_zz as
    REDFT01 of -scale q_a^2 psihat, d_t psi = REDFT01 of scale (aLin psihat + Nhat)."""
    psi = orc.psi
    psiq = dct3d(psi)
    nq = dct3d(orc._nonlin_local(psi))
    s = orc.scale
    return {"dxx": idct3d(-s * orc.qx ** 2 * psiq), "dyy": idct3d(-s * orc.qy ** 2 * psiq),
            "dzz": idct3d(-s * orc.qz ** 2 * psiq), "dt": idct3d(s * (orc.a_lin * psiq + nq))}


def neumann_spectral_derivatives(psi, dx: float):
    """First and mixed derivatives of the cosine series of psi (the REDFT01
    expansion of scale REDFT10(psi)), exactly: d/dx turns the cosine series in x
    into the sine series RODFT01 of X[m] = -q_{m+1} A[m+1] (m < N-1; X[N-1] = 0).
    Returns psi_x, psi_y, psi_z, psi_xy, psi_xz, psi_yz."""
    n = psi.shape[0]
    a = dct3d(psi) / (8.0 * n ** 3)
    q = kvec_dct(n, dx)

    def dsin(b, ax):
        b = np.moveaxis(b, ax, 0)
        out = np.zeros_like(b)
        out[:-1] = -q[1:].reshape((-1,) + (1,) * (b.ndim - 1)) * b[1:]
        return np.moveaxis(out, 0, ax)

    def inv(b, sine_axes):
        for ax in range(3):
            b = (sfft.dst if ax in sine_axes else sfft.dct)(b, type=3, axis=ax, workers=WORKERS)
        return b

    ax_, ay_, az_ = dsin(a, 0), dsin(a, 1), dsin(a, 2)
    return (inv(ax_, (0,)), inv(ay_, (1,)), inv(az_, (2,)), inv(dsin(ax_, 1), (0, 1)), inv(dsin(ax_, 2), (0, 2)),
            inv(dsin(ay_, 2), (1, 2)))


def neumann_curvature_scan(psi, f, dx: float, threshold: float = 0.7, spectral=None):
    """Column scan of the Neumann curvature pass (cosNoAdvMorphCurv.cpp:874-965).

    For each (i, j) scan -z from the top for the first psi < 0 after
    psi > threshold; move up one voxel (k2 = k + 1) when that one is closer to
    zero.  At k2: |grad psi| from wall-one-sided centred differences, v_n =
    d_t psi / |grad psi|, mixed derivatives as differences of the gradient
    (psi_xy along y at k2; psi_xz, psi_yz along z, formula chosen by k as the
    reference does), and Megrabov's H (/|grad psi|^3) and K (/|grad psi|^4).
    The x gradient is taken from the current psi (the reference's rank-0 copy
    of psi can be stale there).  Where the reference's z formula would read
    past the top of the column (k2 = N-1 with k interior) the one-sided
    backward formula is used.  Returns z = k2, v_n, H, K (-1 / NaN when no
    crossing).  ``spectral`` (neumann_spectral_derivatives(psi, dx)) replaces
    the difference gradient and mixed derivatives by the exact ones of the
    cosine series."""
    n = psi.shape[0]
    gx, gy = _fd_wall(psi, 0, dx), _fd_wall(psi, 1, dx)
    gz = _fd_wall(psi, 2, dx)
    if spectral is not None:
        gx, gy, gz = spectral[:3]
    td = 2 * dx
    z = -np.ones((n, n), dtype=np.int64)
    vn = np.full((n, n), np.nan)
    hh = np.full((n, n), np.nan)
    kk = np.full((n, n), np.nan)
    for i in range(n):
        for j in range(n):
            col = psi[i, j]
            track = 0
            for k in range(n - 1, -1, -1):
                if col[k] > threshold and track == 0:
                    track = 1
                if col[k] < 0 and track == 1:
                    k2 = k + 1 if abs(col[k]) > abs(col[k + 1]) else k
                    Gx, Gy, Gz = gx[i, j, k2], gy[i, j, k2], gz[i, j, k2]
                    g = np.sqrt(Gx * Gx + Gy * Gy + Gz * Gz)
                    if 0 < j < n - 1:
                        dxy = (gx[i, j + 1, k2] - gx[i, j - 1, k2]) / td
                    elif j == 0:
                        dxy = 2 * (gx[i, 1, k2] - gx[i, 0, k2]) / td
                    else:
                        dxy = 2 * (gx[i, j, k2] - gx[i, j - 1, k2]) / td
                    if 0 < k < n - 1 and k2 + 1 < n:
                        dxz = (gx[i, j, k2 + 1] - gx[i, j, k2 - 1]) / td
                        dyz = (gy[i, j, k2 + 1] - gy[i, j, k2 - 1]) / td
                    elif k == 0:
                        dxz = 2 * (gx[i, j, k2 + 1] - gx[i, j, k2]) / td
                        dyz = 2 * (gy[i, j, k2 + 1] - gy[i, j, k2]) / td
                    else:
                        dxz = 2 * (gx[i, j, k2] - gx[i, j, k2 - 1]) / td
                        dyz = 2 * (gy[i, j, k2] - gy[i, j, k2 - 1]) / td
                    if spectral is not None:
                        dxy, dxz, dyz = spectral[3][i, j, k2], spectral[4][i, j, k2], spectral[5][i, j, k2]
                    xx, yy, zz = f["dxx"][i, j, k2], f["dyy"][i, j, k2], f["dzz"][i, j, k2]
                    z[i, j] = k2
                    vn[i, j] = f["dt"][i, j, k2] / g
                    hh[i, j] = ((Gy ** 2 + Gz ** 2) * xx + (Gx ** 2 + Gz ** 2) * yy + (Gx ** 2 + Gy ** 2) * zz
                                - 2 * (Gx * Gy * dxy + Gx * Gz * dxz + Gy * Gz * dyz)) / g ** 3
                    kk[i, j] = (Gz ** 2 * (xx * yy - dxy ** 2) + Gx ** 2 * (yy * zz - dyz ** 2)
                                + Gy ** 2 * (xx * zz - dxz ** 2)
                                + 2 * (Gy * dxy * (Gz * dxz - Gx * zz) + Gx * dxz * (Gy * dyz - Gz * yy)
                                       + Gz * dyz * (Gx * dxy - Gy * xx))) / g ** 4
                    break
    return z, vn, hh, kk


def _trapz(nstart, nend, h, vals):
    """trapz of morphSurfAmp.cpp:76-86: 0.5 h sum_{n < nend - nstart} (v[n] + v[n+1])."""
    t = 0.0
    for m in range(nend - nstart):
        t += vals[m] + vals[m + 1]
    return 0.5 * h * t


def local_amplitude_direct(psi, dx: float, nw: int, q0: float = 1.0):
    """psiAvg of morphSurfAmp.cpp:1005-1125, loop for loop (small grids only)."""
    n = psi.shape[0]
    nl = nw // 2

    def box(i0, i1, j0, j1, k0, k1):
        az = []
        for k2 in range(k0, k1 + 1):
            ay = []
            for j2 in range(j0, j1 + 1):
                ax = [psi[i2, j2, k2] ** 2 for i2 in range(i0, i1 + 1)]
                ay.append(_trapz(i0, i1, dx, ax))
            az.append(_trapz(j0, j1, dx, ay))
        return _trapz(k0, k1, dx, az)

    ref = box(nl, 3 * nl, nl, 3 * nl, nl, 3 * nl)
    lam3 = (2 * np.pi / q0) ** 3
    out = np.empty_like(psi)
    for i in range(n):
        i0, i1 = max(i - nl, 0), min(i + nl, n - 1)
        for j in range(n):
            j0, j1 = max(j - nl, 0), min(j + nl, n - 1)
            for k in range(n):
                k0, k1 = max(k - nl, 0), min(k + nl, n - 1)
                vol = (i1 - i0) * dx * (j1 - j0) * dx * (k1 - k0) * dx
                out[i, j, k] = box(i0, i1, j0, j1, k0, k1) / (ref * vol / lam3)
    return out


def _window_trapz(f, axis, nl, h):
    """Clipped-window trapezoid along ``axis``: h (sum f[a..b] - (f[a] + f[b]) / 2),
    a = max(0, p - nl), b = min(n - 1, p + nl)."""
    f = np.moveaxis(f, axis, 0)
    n = f.shape[0]
    c = np.concatenate([np.zeros((1,) + f.shape[1:]), np.cumsum(f, axis=0)])
    p = np.arange(n)
    a, b = np.maximum(p - nl, 0), np.minimum(p + nl, n - 1)
    return np.moveaxis(h * (c[b + 1] - c[a] - 0.5 * (f[a] + f[b])), 0, axis)


def local_amplitude(psi, dx: float, nw: int, q0: float = 1.0):
    """psiAvg of morphSurfAmp.cpp:1005-1125 through the separable form of its
    nested trapezoids (the box is a product domain); equals
    local_amplitude_direct up to rounding."""
    n = psi.shape[0]
    nl = nw // 2
    t = _window_trapz(_window_trapz(_window_trapz(psi * psi, 0, nl, dx), 1, nl, dx), 2, nl, dx)
    ref = t[2 * nl, 2 * nl, 2 * nl]
    p = np.arange(n)
    ln = (np.minimum(p + nl, n - 1) - np.maximum(p - nl, 0)) * dx
    vol = ln[:, None, None] * ln[None, :, None] * ln[None, None, :]
    return t / (ref * vol / (2 * np.pi / q0) ** 3)


# ---------------------------------------------------------------------------
# diagnostics
# ---------------------------------------------------------------------------

def l1_monitor(psi_new, psi_old, dt):
    """L1 = sum|psiNew - psi| / (dt sum|psiNew|) (periodicFFT/pf3d.cpp:489-509)."""
    return float(np.abs(psi_new - psi_old).sum() / (dt * np.abs(psi_new).sum()))


def _local_density(psi, p: Params):
    if p.nonlinearity == "quintic":
        pot = -0.25 * p.beta * psi ** 4 + p.gamma / 6.0 * psi ** 6
    else:
        pot = -p.beta / 3.0 * psi ** 3 + 0.25 * p.gamma * psi ** 4
    return -0.5 * p.eps * psi * psi + pot


def energy_spectral_periodic(psi, p: Params) -> float:
    """Lyapunov functional with the exact (spectral) Laplacian.

    F = dV sum[-eps/2 psi^2 + alpha/2 ((q0^2+lap) psi)^2 - beta/4 psi^4
    + gamma/6 psi^6], the density of energyPsi.m:225-228 with the periodic
    sum of the grid in place of trapz and FD.
    """
    n = psi.shape[0]
    dv = p.dx ** 3
    q = kvec_periodic(n, p.dx)
    mq2 = q[:, None, None] ** 2 + q[None, :, None] ** 2 + q[None, None, :] ** 2
    ph = sfft.fftn(psi, workers=WORKERS)
    grad_term = 0.5 * p.alpha * (np.abs(ph) ** 2 * (p.q0 ** 2 - mq2) ** 2).sum() / n ** 3
    return float(dv * (_local_density(psi, p).sum() + grad_term))


def energy_spectral_neumann(psi, p: Params) -> float:
    """Same functional with the DCT (Neumann) Laplacian.

    Parseval for REDFT10: sum x^2 = (1/2N) (X0^2/2 + sum_{k>0} Xk^2) per axis.
    """
    n = psi.shape[0]
    dv = p.dx ** 3
    q = kvec_dct(n, p.dx)
    mq2 = q[:, None, None] ** 2 + q[None, :, None] ** 2 + q[None, None, :] ** 2
    x = dct3d(psi)
    w = np.ones(n)
    w[0] = 0.5
    wt = w[:, None, None] * w[None, :, None] * w[None, None, :] / (2.0 * n) ** 3
    grad_term = 0.5 * p.alpha * (wt * x * x * (p.q0 ** 2 - mq2) ** 2).sum()
    return float(dv * (_local_density(psi, p).sum() + grad_term))


def energy_fd_trapz(psi, p: Params) -> float:
    """energyPsi.m:131-234 restated: periodic 2nd-order FD Laplacian (:217-219),
    density (:225-228), triple trapz over xV = 0:dx:L-dx (:234)."""
    dx2 = 1.0 / p.dx ** 2
    lap = (np.roll(psi, 1, 0) + np.roll(psi, -1, 0) + np.roll(psi, 1, 1) + np.roll(psi, -1, 1)
           + np.roll(psi, 1, 2) + np.roll(psi, -1, 2) - 6.0 * psi) * dx2
    dens = _local_density(psi, p) + 0.5 * p.alpha * (p.q0 ** 2 * psi + lap) ** 2
    e = np.trapezoid(dens, dx=p.dx, axis=2)
    e = np.trapezoid(e, dx=p.dx, axis=1)
    e = np.trapezoid(e, dx=p.dx, axis=0)
    return float(e)


def dominant_wavenumber(psi, dx: float) -> float:
    """|q| of the shell (width 2 pi/L) holding the most spectral power, DC excluded."""
    n = psi.shape[0]
    q = kvec_periodic(n, dx)
    mq = np.sqrt(q[:, None, None] ** 2 + q[None, :, None] ** 2 + q[None, None, : n // 2 + 1] ** 2)
    ph = np.abs(r2c(psi)) ** 2
    w = np.full(n // 2 + 1, 2.0)
    w[0] = 1.0
    w[n // 2] = 1.0
    ph = ph * w[None, None, :]
    dq = 2.0 * np.pi / (n * dx)
    shell = np.rint(mq / dq).astype(np.int64)
    power = np.bincount(shell.ravel(), weights=ph.ravel())
    power[0] = 0.0
    return float(np.argmax(power) * dq)


def dominant_wavenumber_neumann(psi, dx: float) -> float:
    """The same shell argmax for the Neumann box: REDFT10 spectrum, q = pi m / L,
    shells of width pi / L, the power of each mode weighted as in Parseval's
    sum of the REDFT10 pair (1/2 on every zero index)."""
    n = psi.shape[0]
    q = kvec_dct(n, dx)
    mq = np.sqrt(q[:, None, None] ** 2 + q[None, :, None] ** 2 + q[None, None, :] ** 2)
    x = dct3d(psi)
    w = np.ones(n)
    w[0] = 0.5
    ph = x * x * (w[:, None, None] * w[None, :, None] * w[None, None, :])
    dq = np.pi / (n * dx)
    shell = np.rint(mq / dq).astype(np.int64)
    power = np.bincount(shell.ravel(), weights=ph.ravel())
    power[0] = 0.0
    return float(np.argmax(power) * dq)


# ---------------------------------------------------------------------------
# discrete adjoint of the plain periodic CNAB2 scheme
# ---------------------------------------------------------------------------

def adjoint_gradients_periodic(psi0, p: Params, steps: int, target):
    """Exact discrete adjoint of ``PeriodicOracle`` (plain, CNAB2, no penalty)
    for L = 1/2 ||psi_T - target||^2 (plain sum over grid points).

    Forward map (real space, A and B symmetric Fourier multipliers):
        psi^{n+1} = A psi^n + B (3 N(psi^n) - N(psi^{n-1})),  N(psi^{-1}) := N(psi^0)
        A = F^-1 diag(C1/C2) F,  B = F^-1 diag(dt/2 / C2) F
    Reverse sweep:
        lam^T = psi^T - target
        lam^n = A lam^{n+1} + N'(psi^n) (c_n B lam^{n+1} - B lam^{n+2}),
        c_n = 3 for n >= 1, c_0 = 2 ; lam^{T+1} = 0.
    Parameter gradients use d psihat^{n+1}/d a = dt/2 (psihat^n + psihat^{n+1}) / C2
    with a = aLin, da/d eps = 1, da/d q0 = 4 alpha q0 (|q|^2 - q0^2).
    Returns (loss, dL/d eps, dL/d q0, dL/d psi0).
    """
    assert p.scheme == "cnab2" and p.w_mid == 0.0
    orc = PeriodicOracle(psi0, p)
    states = [orc.psi.copy()]
    for _ in range(steps):
        states.append(orc.step().copy())
    n = p.n
    lam_next = states[-1] - target
    loss = 0.5 * float((lam_next ** 2).sum())
    a_mul = orc.c1 / orc.c2
    b_mul = 0.5 * p.dt / orc.c2
    da_dq0 = 4.0 * p.alpha * p.q0 * (orc.mq2 - p.q0 ** 2)
    w = np.full(n // 2 + 1, 2.0)
    w[0] = 1.0
    w[n // 2] = 1.0
    w = w[None, None, :]
    g_eps = 0.0
    g_q0 = 0.0
    blam_next2 = np.zeros((n, n, n))   # B lam^{n+2}
    for k in range(steps - 1, -1, -1):
        # lam_next = lam^{k+1}; states[k] = psi^k
        lq = r2c(lam_next)
        ph_k = r2c(states[k])
        ph_k1 = r2c(states[k + 1])
        dpar = 0.5 * p.dt * (ph_k + ph_k1) / orc.c2
        # <lam, F^-1 X> = (1/N^3) sum_k w conj(lamhat) X  (real)
        inner = (w * np.conj(lq) * dpar).real / n ** 3
        g_eps += float(inner.sum())
        g_q0 += float((inner * da_dq0).sum())
        blam = c2r(orc.scale * b_mul * lq, n)
        alam = c2r(orc.scale * a_mul * lq, n)
        c = 3.0 if k >= 1 else 2.0
        lam_k = alam + nonlin_deriv(states[k], p) * (c * blam - blam_next2)
        blam_next2 = blam
        lam_next = lam_k
    return loss, g_eps, g_q0, lam_next
