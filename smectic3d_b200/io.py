"""The reference's text file formats.

psi files (psi.dat, psiIC.dat, psiB.dat): N^3 values, i, j, k order with k
fastest, each followed by "\\n " (periodicFFT/pf3d.cpp:534-540); the
reference writes them with ostream's default 6 significant digits.
L1.dat: one value per line (periodicFFT/pf3d.cpp:510-512).
surfTrack files (surfPsi.dat, velSurf.dat, curvH.dat, curvK.dat): one value
per found column in (i, j) order, each followed by "\\n "
(periodicFFT/surfTrack.cpp:787-799).
"""
from __future__ import annotations

import os

import numpy as np


def write_psi_text(path, psi: np.ndarray, digits: int | None = None) -> None:
    """digits=None: exact (17 significant digits); 6 reproduces the reference."""
    fmt = "%.17g" if digits is None else f"%.{digits}g"
    flat = np.ascontiguousarray(psi, dtype=np.float64).ravel()
    with open(path, "w") as f:
        f.write("".join((fmt % v) + "\n " for v in flat))


def read_psi_text(path, n: int) -> np.ndarray:
    data = np.fromstring(open(path).read(), sep=" ") if os.path.getsize(path) else np.empty(0)
    if data.size < n ** 3:
        raise ValueError(f"{path}: {data.size} values, expected {n ** 3}")
    return data[: n ** 3].reshape(n, n, n)


def read_l1(path) -> np.ndarray:
    return np.loadtxt(path, ndmin=1) if os.path.getsize(path) else np.empty(0)


def write_surface_files(directory, z, vn, hh, kk) -> int:
    """Write the four surfTrack files for the columns where a crossing exists;
    returns how many."""
    found = np.asarray(z) >= 0
    cols = {"surfPsi.dat": np.asarray(z)[found], "velSurf.dat": np.asarray(vn)[found],
            "curvH.dat": np.asarray(hh)[found], "curvK.dat": np.asarray(kk)[found]}
    for name, vals in cols.items():
        with open(os.path.join(directory, name), "w") as f:
            if name == "surfPsi.dat":
                f.write("".join(f"{int(v)}\n " for v in vals))
            else:
                f.write("".join(f"{v:.6g}\n " for v in vals))
    return int(found.sum())
