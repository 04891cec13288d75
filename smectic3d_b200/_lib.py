"""ctypes binding of ``libsmectic_b200.so`` (declarations: include/smectic_b200.h).

The library is the only compute path: if it is missing, importing anything that
needs it raises, with no fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libsmectic_b200.so"

SH_OK, SH_EINVAL, SH_ENOMEM, SH_ENONFINITE, SH_ETIMEOUT, SH_ECUDA, SH_EUNSUPPORTED, SH_ESTATE = range(8)
SH_PERIODIC, SH_NEUMANN = 0, 1
SH_QUINTIC, SH_QUAD_CUBIC = 0, 1
SH_CNAB2, SH_IMEX_EULER = 0, 1
SH_FP64, SH_FP32, SH_FP32_UPDATE64 = 0, 1, 2
SH_LAYOUT_DENSE, SH_LAYOUT_PADDED = 0, 1
SH_CURV_DIFFERENCE, SH_CURV_SPECTRAL = 0, 1

# every entry point include/smectic_b200.h declares
EXPORTS = (
    "sh_default_params", "sh_create", "sh_destroy", "sh_set_psi", "sh_set_psi_device", "sh_get_psi",
    "sh_get_psi_device", "sh_step", "sh_step_async", "sh_prepare", "sh_run", "sh_energy", "sh_dominant_wavenumber", "sh_velocity", "sh_energy_trace", "sh_l1",
    "sh_surface_step", "sh_local_amplitude", "sh_adjoint", "sh_adjoint_forward", "sh_adjoint_backward", "sh_checkpoint_save", "sh_checkpoint_load", "sh_host_alloc", "sh_host_free",
    "sh_l1_noalloc", "sh_profile_steps", "sh_residency", "sh_synchronize", "sh_stream", "sh_steps_taken", "sh_kernel_launches", "sh_last_error", "sh_version",
)


class ShParams(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("batch", C.c_int), ("boundary", C.c_int), ("advection", C.c_int),
        ("nonlinearity", C.c_int), ("scheme", C.c_int), ("precision", C.c_int), ("l1_interval", C.c_int),
        ("energy_trace", C.c_int), ("variant", C.c_int),
        ("dx", C.c_double), ("dt", C.c_double), ("eps", C.c_double), ("beta", C.c_double),
        ("gamma", C.c_double), ("alpha", C.c_double), ("q0", C.c_double), ("eta", C.c_double),
        ("rho", C.c_double), ("w_mid", C.c_double), ("sub_sigma", C.c_double), ("sub_z0", C.c_double),
        ("eps_per_replica", C.POINTER(C.c_double)), ("curvature", C.c_int), ("replica_block", C.c_int),
        ("pencil_tile", C.c_int),
    ]


class ShError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"smectic_b200 error {code}: {msg}")
        self.code = code


_lib = None


def load() -> C.CDLL:
    """Load the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: run `python -m smectic3d_b200.build` (or __graft_entry__.build())")
    lib = C.CDLL(os.fspath(LIB_PATH))
    vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
    sig = {
        "sh_default_params": (C.c_int, [C.POINTER(ShParams)]),
        "sh_create": (C.c_int, [C.POINTER(ShParams), C.POINTER(vp)]),
        "sh_destroy": (C.c_int, [vp]),
        "sh_set_psi": (C.c_int, [vp, vp, C.c_int]),
        "sh_set_psi_device": (C.c_int, [vp, vp]),
        "sh_get_psi": (C.c_int, [vp, vp, C.c_int]),
        "sh_get_psi_device": (C.c_int, [vp, vp]),
        "sh_step": (C.c_int, [vp, C.c_int]),
        "sh_step_async": (C.c_int, [vp, C.c_int]),
        "sh_prepare": (C.c_int, [vp]),
        "sh_run": (C.c_int, [vp, vp, C.c_int, vp, C.c_int]),
        "sh_energy": (C.c_int, [vp, dp]),
        "sh_dominant_wavenumber": (C.c_int, [vp, dp]),
        "sh_velocity": (C.c_int, [vp, vp, vp, vp]),
        "sh_energy_trace": (C.c_int, [vp, dp, C.c_int, ip]),
        "sh_l1": (C.c_int, [vp, dp, ip]),
        "sh_surface_step": (C.c_int, [vp, ip, dp, dp, dp]),
        "sh_local_amplitude": (C.c_int, [vp, C.c_int, dp]),
        "sh_adjoint": (C.c_int, [vp, vp, C.c_int, vp, C.c_int, dp, dp, vp]),
        "sh_adjoint_forward": (C.c_int, [vp, vp, C.c_int, C.c_int]),
        "sh_adjoint_backward": (C.c_int, [vp, vp, dp, dp, vp]),
        "sh_checkpoint_save": (C.c_int, [vp, vp, C.POINTER(C.c_size_t)]),
        "sh_checkpoint_load": (C.c_int, [vp, vp, C.c_size_t]),
        "sh_host_alloc": (C.c_int, [C.c_size_t, C.POINTER(vp)]),
        "sh_host_free": (C.c_int, [vp]),
        "sh_l1_noalloc": (C.c_int, [vp, vp, C.c_longlong, C.c_int, C.c_double, vp, vp]),
        "sh_profile_steps": (C.c_int, [vp, C.c_int, dp, dp]),
        "sh_synchronize": (C.c_int, [vp]),
        "sh_stream": (vp, [vp]),
        "sh_steps_taken": (C.c_longlong, [vp]),
        "sh_kernel_launches": (C.c_int, [vp, C.POINTER(C.c_longlong)]),
        "sh_residency": (C.c_int, [vp, C.POINTER(C.c_int)]),
        "sh_last_error": (C.c_char_p, [vp]),
        "sh_version": (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(rc: int, handle=None) -> None:
    if rc != SH_OK:
        lib = load()
        msg = lib.sh_last_error(handle)
        raise ShError(rc, msg.decode() if msg else "")
