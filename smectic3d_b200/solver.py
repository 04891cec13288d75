"""Python mirror of the reference's time-loop interface over the C-ABI.

``Params`` carries the constants the reference hard-codes in main()
(periodicFFT/pf3d.cpp:35-73, cosFFT/mesabi/cosNoAdvMorph.cpp:74-112) and
``Solver`` runs the loop body (periodicFFT/pf3d.cpp:390-550) on the GPU.
Arrays cross the boundary as float64 in the reference's index order
(i, j, k with k fastest).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math

import numpy as np

from . import _lib as L


@dataclasses.dataclass
class Params:
    n: int = 128
    batch: int = 1
    boundary: str = "periodic"       # "periodic" (R2C/C2R) or "neumann" (REDFT10/REDFT01)
    advection: bool = False
    nonlinearity: str = "quintic"    # beta psi^3 - gamma psi^5 (reference) | "quad_cubic"
    scheme: str = "cnab2"            # reference CN + AB2 | "imex_euler"
    precision: str = "fp64"          # "fp64" | "fp32" | "fp32_u64" (FP32 fields, FP64 CNAB2 update)
    l1_interval: int = 0             # 100 in the reference (periodicFFT/pf3d.cpp:489)
    energy_trace: bool = False
    dx: float = 2.0 * math.pi / 8.0
    dt: float = 0.05
    eps: float = -0.75
    beta: float = 2.0
    gamma: float = 1.0
    alpha: float = 1.0
    q0: float = 1.0
    eta: float = 1.0
    rho: float = 1.0
    w_mid: float = 0.0
    sub_sigma: float = 0.0
    sub_z0: float = 1e-4
    eps_per_replica: tuple | None = None
    variant: int = 0                 # plane-pass cluster size (0 = default, -1 = autotune)
    curvature: str = "difference"    # Neumann curvature pass: "difference" (reference) | "spectral"
    replica_block: int = 0           # batched plain steps: replicas per L2-resident block (0 = off)
    pencil_tile: int = 0             # lines per pencil CTA (0 = default; 8, 16, 32 at 64^3 and 128^3)

    @staticmethod
    def from_nw(n: int, nw: int, q0: float = 1.0, **kw) -> "Params":
        """dx from points per wavelength, as the reference does: L = N 2 pi/(q0 Nw)."""
        return Params(n=n, dx=2.0 * math.pi / (q0 * nw), q0=q0, **kw)

    def to_c(self):
        p = L.ShParams()
        p.n, p.batch = self.n, self.batch
        p.boundary = {"periodic": L.SH_PERIODIC, "neumann": L.SH_NEUMANN}[self.boundary]
        p.advection = int(bool(self.advection))
        p.nonlinearity = {"quintic": L.SH_QUINTIC, "quad_cubic": L.SH_QUAD_CUBIC}[self.nonlinearity]
        p.scheme = {"cnab2": L.SH_CNAB2, "imex_euler": L.SH_IMEX_EULER}[self.scheme]
        p.precision = {"fp64": L.SH_FP64, "fp32": L.SH_FP32, "fp32_u64": L.SH_FP32_UPDATE64}[self.precision]
        p.l1_interval = self.l1_interval
        p.energy_trace = int(bool(self.energy_trace))
        p.variant = int(self.variant)
        p.curvature = {"difference": L.SH_CURV_DIFFERENCE, "spectral": L.SH_CURV_SPECTRAL}[self.curvature]
        p.replica_block = int(self.replica_block)
        p.pencil_tile = int(self.pencil_tile)
        for k in ("dx", "dt", "eps", "beta", "gamma", "alpha", "q0", "eta", "rho", "w_mid", "sub_sigma", "sub_z0"):
            setattr(p, k, float(getattr(self, k)))
        keep = None
        if self.eps_per_replica is not None:
            keep = (C.c_double * self.batch)(*[float(e) for e in self.eps_per_replica])
            p.eps_per_replica = C.cast(keep, C.POINTER(C.c_double))
        return p, keep


class Solver:
    """One GPU solver handle (all replicas of ``params.batch``)."""

    def __init__(self, params: Params):
        self.lib = L.load()
        if params.variant < 0:
            from .autotune import best_shape
            params = dataclasses.replace(params, **best_shape(dataclasses.replace(params, variant=0)))
        self.params = params
        cp, keep = params.to_c()
        h = C.c_void_p()
        L.check(self.lib.sh_create(C.byref(cp), C.byref(h)), None)
        self.h = h
        self._keep = keep
        n = params.n
        self.shape = (params.batch, n, n, n) if params.batch > 1 else (n, n, n)

    def close(self):
        if getattr(self, "h", None):
            self.lib.sh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _chk(self, rc):
        L.check(rc, self.h)

    # -- state ---------------------------------------------------------------
    def set_psi(self, psi: np.ndarray, layout: int = L.SH_LAYOUT_DENSE):
        a = np.ascontiguousarray(psi, dtype=np.float64)
        self._chk(self.lib.sh_set_psi(self.h, a.ctypes.data, layout))

    def get_psi(self, layout: int = L.SH_LAYOUT_DENSE) -> np.ndarray:
        n, b = self.params.n, self.params.batch
        if layout == L.SH_LAYOUT_DENSE:
            out = np.empty(self.shape, dtype=np.float64)
        else:
            out = np.empty((b, n, n, 2 * (n // 2 + 1)) if b > 1 else (n, n, 2 * (n // 2 + 1)), dtype=np.float64)
        self._chk(self.lib.sh_get_psi(self.h, out.ctypes.data, layout))
        return out

    def set_psi_device(self, ptr: int):
        self._chk(self.lib.sh_set_psi_device(self.h, C.c_void_p(ptr)))

    def get_psi_device(self, ptr: int):
        self._chk(self.lib.sh_get_psi_device(self.h, C.c_void_p(ptr)))

    def step(self, nsteps: int = 1):
        self._chk(self.lib.sh_step(self.h, int(nsteps)))

    def step_async(self, nsteps: int = 1):
        self._chk(self.lib.sh_step_async(self.h, int(nsteps)))

    def prepare(self):
        """Instantiate the replayed step graph now (runs nothing)."""
        self._chk(self.lib.sh_prepare(self.h))

    def run(self, psi0: np.ndarray, nsteps: int, out: np.ndarray | None = None) -> np.ndarray:
        a = np.ascontiguousarray(psi0, dtype=np.float64)
        if out is None:
            out = np.empty(self.shape, dtype=np.float64)
        self._chk(self.lib.sh_run(self.h, a.ctypes.data, int(nsteps), out.ctypes.data, L.SH_LAYOUT_DENSE))
        return out

    def profile_steps(self, nsteps: int):
        """Per-pass device time (ms) of ``nsteps`` steps: (pencil, plane)."""
        a, b = C.c_double(), C.c_double()
        self._chk(self.lib.sh_profile_steps(self.h, int(nsteps), C.byref(a), C.byref(b)))
        return a.value, b.value

    def residency(self) -> dict:
        """CTAs per SM and waves of the two step kernels on this GPU."""
        o = (C.c_int * 7)()
        self._chk(self.lib.sh_residency(self.h, o))
        plane_res = o[1] * o[2]
        return {"plane_ctas_per_sm": o[0], "plane_clusters_resident": o[1], "plane_cluster": o[2],
                "plane_ctas": o[3], "plane_waves": o[3] / plane_res if plane_res else None,
                "pencil_ctas_per_sm": o[4], "pencil_ctas": o[5],
                "pencil_waves": o[5] / (o[4] * o[6]) if o[4] else None, "sms": o[6]}

    def synchronize(self):
        self._chk(self.lib.sh_synchronize(self.h))

    @property
    def stream(self) -> int:
        return self.lib.sh_stream(self.h) or 0

    @property
    def steps_taken(self) -> int:
        return int(self.lib.sh_steps_taken(self.h))

    @property
    def kernel_launches(self) -> int:
        c = C.c_longlong()
        self._chk(self.lib.sh_kernel_launches(self.h, C.byref(c)))
        return int(c.value)

    # -- diagnostics -----------------------------------------------------------
    def energy(self) -> np.ndarray:
        out = np.empty(self.params.batch, dtype=np.float64)
        self._chk(self.lib.sh_energy(self.h, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def dominant_wavenumber(self) -> np.ndarray:
        """|q| of the spectral shell with the most power, per replica."""
        out = np.empty(self.params.batch, dtype=np.float64)
        self._chk(self.lib.sh_dominant_wavenumber(self.h, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def velocity(self):
        """(u_x, u_y, u_z) of the current state of an advected handle."""
        out = [np.empty(self.shape, dtype=np.float64) for _ in range(3)]
        self._chk(self.lib.sh_velocity(self.h, *(o.ctypes.data for o in out)))
        return tuple(out)

    def energy_trace(self) -> np.ndarray:
        cnt = C.c_int()
        self._chk(self.lib.sh_energy_trace(self.h, None, 0, C.byref(cnt)))
        out = np.empty((cnt.value, self.params.batch), dtype=np.float64)
        if cnt.value:
            self._chk(self.lib.sh_energy_trace(self.h, out.ctypes.data_as(C.POINTER(C.c_double)), cnt.value,
                                               C.byref(cnt)))
        return out

    def l1(self):
        out = np.empty(self.params.batch, dtype=np.float64)
        cnt = C.c_int()
        self._chk(self.lib.sh_l1(self.h, out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(cnt)))
        return out, cnt.value

    def surface_step(self):
        """Surface pass and one step; per (x, y) column the crossing z (-1 if
        none), v_n, H and K (NaN if none).  Periodic advected handles run
        surfTrack on the new psi; Neumann handles run the curvature pass
        (Megrabov H and K) on the psi before the step."""
        n, b = self.params.n, self.params.batch
        shape = (b, n, n) if b > 1 else (n, n)
        z = np.empty(shape, dtype=np.int32)
        vn = np.empty(shape, dtype=np.float64)
        hh = np.empty(shape, dtype=np.float64)
        kk = np.empty(shape, dtype=np.float64)
        self._chk(self.lib.sh_surface_step(self.h, z.ctypes.data_as(C.POINTER(C.c_int)),
                                           vn.ctypes.data_as(C.POINTER(C.c_double)),
                                           hh.ctypes.data_as(C.POINTER(C.c_double)),
                                           kk.ctypes.data_as(C.POINTER(C.c_double))))
        return z, vn, hh, kk

    def local_amplitude(self, nw: int) -> np.ndarray:
        """Local-amplitude map psiAvg of the current psi (morphSurfAmp.cpp:1005-1125),
        the same shape as get_psi()."""
        out = np.empty(self.shape, dtype=np.float64)
        self._chk(self.lib.sh_local_amplitude(self.h, int(nw), out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def adjoint(self, psi0: np.ndarray, nsteps: int, dl_dpsi_t: np.ndarray, ckpt_every: int = 50):
        """Discrete adjoint of the CNAB2 loop: returns (dL/d eps, dL/d q0, dL/d psi0)
        per replica for a loss with gradient dl_dpsi_t at psi^T."""
        a = np.ascontiguousarray(psi0, dtype=np.float64)
        g = np.ascontiguousarray(dl_dpsi_t, dtype=np.float64)
        b = self.params.batch
        ge = np.empty(b, dtype=np.float64)
        gq = np.empty(b, dtype=np.float64)
        gp = np.empty(self.shape, dtype=np.float64)
        self._chk(self.lib.sh_adjoint(self.h, a.ctypes.data, int(nsteps), g.ctypes.data, int(ckpt_every),
                                      ge.ctypes.data_as(C.POINTER(C.c_double)),
                                      gq.ctypes.data_as(C.POINTER(C.c_double)), gp.ctypes.data))
        return ge, gq, gp

    def adjoint_forward(self, psi0: np.ndarray, nsteps: int, ckpt_every: int = 50):
        """nsteps steps from psi0 keeping the adjoint's checkpoints; the handle
        is left at psi^T (read it with get_psi)."""
        a = np.ascontiguousarray(psi0, dtype=np.float64)
        self._chk(self.lib.sh_adjoint_forward(self.h, a.ctypes.data, int(nsteps), int(ckpt_every)))

    def adjoint_backward(self, dl_dpsi_t: np.ndarray):
        """Reverse sweep from the checkpoints of the last adjoint_forward:
        (dL/d eps, dL/d q0, dL/d psi0) per replica."""
        g = np.ascontiguousarray(dl_dpsi_t, dtype=np.float64)
        b = self.params.batch
        ge = np.empty(b, dtype=np.float64)
        gq = np.empty(b, dtype=np.float64)
        gp = np.empty(self.shape, dtype=np.float64)
        self._chk(self.lib.sh_adjoint_backward(self.h, g.ctypes.data, ge.ctypes.data_as(C.POINTER(C.c_double)),
                                               gq.ctypes.data_as(C.POINTER(C.c_double)), gp.ctypes.data))
        return ge, gq, gp

    def checkpoint(self) -> bytes:
        size = C.c_size_t()
        self._chk(self.lib.sh_checkpoint_save(self.h, None, C.byref(size)))
        buf = (C.c_char * size.value)()
        self._chk(self.lib.sh_checkpoint_save(self.h, buf, C.byref(size)))
        return bytes(buf)

    def restore(self, blob: bytes):
        buf = (C.c_char * len(blob)).from_buffer_copy(blob)
        self._chk(self.lib.sh_checkpoint_load(self.h, buf, len(blob)))
