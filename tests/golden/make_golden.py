"""Generate the golden vectors under tests/golden/ from the FP64 oracle.

    python -m tests.golden.make_golden            # the small cases
    python -m tests.golden.make_golden --full     # the measurement configurations (about 25 min)

Each case stores its inputs (psi0, parameters) and the oracle's outputs, so
the GPU parity tests compare against fixed numbers that do not depend on the
oracle being importable or on SciPy's version.  The reference itself cannot
be run here (it needs FFTW-MPI and MPI), so these vectors come from the
oracle, whose pins are the analytic tests in tests/test_oracle.py.
"""
from __future__ import annotations

import dataclasses
import math
import os

import numpy as np

from oracle import sh_oracle as O
from smectic3d_b200 import ic

HERE = os.path.dirname(os.path.abspath(__file__))


def path(name: str) -> str:
    return os.path.join(HERE, name + ".npz")


def _pack(p: O.Params, **arrays):
    d = {k: np.asarray(v) for k, v in arrays.items()}
    for f in dataclasses.fields(p):
        v = getattr(p, f.name)
        d["param_" + f.name] = np.asarray(v)
    return d


def periodic_plain():
    n = 16
    p = O.Params(n=n, dt=0.05)
    psi0 = ic.noise(n, 0) + 1.2 * np.cos(np.arange(n) * p.dx)[None, None, :]
    o = O.PeriodicOracle(psi0, p)
    e0 = O.energy_spectral_periodic(psi0, p)
    o.run(10)
    return _pack(p, psi0=psi0, psi=o.psi, steps=10, energy0=e0, energy=O.energy_spectral_periodic(o.psi, p))


def periodic_lamellae_ref_ic():
    n = 32
    p = O.Params(n=n, dx=2 * math.pi / 16, dt=0.01, eps=-0.7)
    psi0 = ic.pf3d_lamellae(n, p.dx)
    o = O.PeriodicOracle(psi0, p)
    o.run(10)
    return _pack(p, psi0=psi0, psi=o.psi, steps=10, energy=O.energy_spectral_periodic(o.psi, p))


def periodic_imex_quadcubic():
    n = 16
    p = O.Params(n=n, dt=0.05, scheme="imex_euler", nonlinearity="quad_cubic", eps=0.2)
    psi0 = ic.noise(n, 3, 0.3)
    o = O.PeriodicOracle(psi0, p)
    o.run(10)
    return _pack(p, psi0=psi0, psi=o.psi, steps=10)


def periodic_penalty():
    n = 16
    p = O.Params(n=n, dt=0.01, w_mid=1.0)
    psi0 = 1.3 * np.cos(np.arange(n) * p.dx)[None, None, :] + ic.noise(n, 4, 0.2)
    o = O.PeriodicOracle(psi0, p)
    o.run(10)
    return _pack(p, psi0=psi0, psi=o.psi, steps=10)


def neumann_hyperboloid():
    n = 16
    p = O.Params(n=n, dt=0.05)
    psi0 = ic.hyperboloid(n, p.dx, r0_cells=5.0, seed=5)
    o = O.NeumannOracle(psi0, p)
    e0 = O.energy_spectral_neumann(psi0, p)
    o.run(10)
    return _pack(p, psi0=psi0, psi=o.psi, steps=10, energy0=e0, energy=O.energy_spectral_neumann(o.psi, p))


def neumann_l1():
    n = 32
    p = O.Params(n=n, dt=0.05, eps=-0.7)
    psi0 = ic.cos_bottom_hyperboloid(n, p.dx)
    o = O.NeumannOracle(psi0, p)
    o.run(19)
    prev = o.psi.copy()
    o.step()
    return _pack(p, psi0=psi0, psi=o.psi, steps=20, l1=O.l1_monitor(o.psi, prev, p.dt))


def periodic_advected():
    n = 16
    p = O.Params(n=n, dt=0.01, eps=-0.7)
    psi0 = ic.pf3d_lamellae(n, p.dx, kmin=1, kmax=15) + ic.noise(n, 6, 0.05)
    o = O.PeriodicOracle(psi0, p, advect=True)
    o.run(10)
    return _pack(p, psi0=psi0, psi=o.psi, steps=10, advect=True, energy=O.energy_spectral_periodic(o.psi, p))


def neumann_substrate():
    # substrate penalty sigma exp(-z/z0) * in-plane Laplacian on the bottom planes
    # (cosFFT/comet/cosNoAdvMorph.cpp:67-74, 591-623)
    n = 16
    p = O.Params(n=n, dt=0.05, sub_sigma=0.5, sub_z0=1.5)
    psi0 = ic.cos_bottom_hyperboloid(n, p.dx) + ic.noise(n, 8, 0.05)
    o = O.NeumannOracle(psi0, p)
    o.run(10)
    return _pack(p, psi0=psi0, psi=o.psi, steps=10)


def _sub(psi):
    """Compact record of a 64^3 state: every 4th point per axis and two global sums."""
    return {"psi_sub": psi[::4, ::4, ::4].copy(), "sum_sq": float(np.sum(psi * psi)),
            "sum_abs": float(np.sum(np.abs(psi)))}


def periodic_plain_64():
    # the initial condition is regenerated by the test from (ic, seed): only outputs are stored
    n = 64
    p = O.Params(n=n, dt=0.05, eps=-0.7)
    psi0 = ic.noise(n, 11, 0.2) + 1.3 * np.cos(np.arange(n) * p.dx)[None, None, :]
    o = O.PeriodicOracle(psi0, p)
    o.run(20)
    return _pack(p, ic_kind="noise11+lamellae1.3", steps=20, **_sub(o.psi))


def neumann_hyperboloid_64():
    n = 64
    p = O.Params(n=n, dt=0.05, eps=-0.7)
    psi0 = ic.hyperboloid(n, p.dx, r0_cells=12.0, seed=12)
    o = O.NeumannOracle(psi0, p)
    o.run(20)
    return _pack(p, ic_kind="hyperboloid12", steps=20, **_sub(o.psi))


CASES = {
    "periodic_plain_16": periodic_plain,
    "periodic_lamellae_32": periodic_lamellae_ref_ic,
    "periodic_imex_quadcubic_16": periodic_imex_quadcubic,
    "periodic_penalty_16": periodic_penalty,
    "neumann_hyperboloid_16": neumann_hyperboloid,
    "neumann_l1_32": neumann_l1,
    "periodic_advected_16": periodic_advected,
    "neumann_substrate_16": neumann_substrate,
    "periodic_plain_64": periodic_plain_64,
    "neumann_hyperboloid_64": neumann_hyperboloid_64,
}


def full_case(name: str) -> dict:
    """A measurement configuration at its own size and length (full_configs.py):
    the oracle state after each check step, subsampled, with its global sums,
    energy and dominant wavenumber; for the advected cases also the surfTrack
    pass of one more step on a subsample of the columns."""
    from tests.golden import full_configs as F
    cfg = F.CASES[name]
    n, stride = cfg["n"], cfg["stride"]
    p = O.Params(n=n, dx=F.DX, dt=cfg["dt"], eps=cfg.get("eps", -0.75))
    psi0 = F.initial_condition(cfg)
    neumann = cfg["boundary"] == "neumann"
    advect = bool(cfg.get("advect", False))
    orc = O.NeumannOracle(psi0, p) if neumann else O.PeriodicOracle(psi0, p, advect=advect)
    efun = O.energy_spectral_neumann if neumann else O.energy_spectral_periodic
    qfun = O.dominant_wavenumber_neumann if neumann else O.dominant_wavenumber
    out = {"checks": np.asarray(cfg["checks"]), "energy_0": efun(psi0, p)}
    done = 0
    for c in cfg["checks"]:
        orc.run(c - done)
        done = c
        psi = orc.psi
        out[f"psi_sub_{c}"] = F.subsample(psi, stride)
        out[f"sum_sq_{c}"] = float(np.sum(psi * psi))
        out[f"sum_abs_{c}"] = float(np.sum(np.abs(psi)))
        out[f"energy_{c}"] = efun(psi, p)
        out[f"qstar_{c}"] = qfun(psi, p.dx)
    if advect:
        orc.step()
        z, vn, hh, kk = O.surface_scan_vec(orc.psi, *orc.surface_fields())
        ss = cfg["surf_stride"]
        out.update(surf_z=z[::ss, ::ss], surf_vn=vn[::ss, ::ss], surf_h=hh[::ss, ::ss], surf_k=kk[::ss, ::ss],
                   psi_sub_surface=F.subsample(orc.psi, stride))
    return _pack(p, **out)


def full_path(name: str) -> str:
    return path("full_" + name)


def main(argv=None):
    import sys
    argv = sys.argv[1:] if argv is None else argv
    if argv and argv[0] == "--full":
        from tests.golden import full_configs as F
        for name in argv[1:] or list(F.CASES):
            np.savez_compressed(full_path(name), **full_case(name))
            print("wrote", full_path(name), flush=True)
        return
    for name, fn in CASES.items():
        np.savez_compressed(path(name), **fn())
        print("wrote", path(name))


if __name__ == "__main__":
    main()
