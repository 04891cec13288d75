"""GPU parity of the CUDA path (through the C-ABI) against the FP64 oracle.

Tolerances (relative L2 of psi): FP64 path <= 1e-10, FP32 path <= 1e-5 after
100 steps, energies to 1e-10 (FP64) / 5e-6 (FP32) relative (the FP32 state carries ~3e-7 relative error and the
functional cancels strongly between its terms).  Small grids are
compared with the oracle run live and with the committed golden vectors; full
sizes (256^3, 512^3) through size-independent properties: the exact linear
growth factor of grid modes, FP32-vs-FP64 agreement, Lyapunov decrease,
replica independence and checkpoint idempotence.
"""
import math
import os

import numpy as np
import pytest

import smectic3d_b200 as S
from smectic3d_b200 import _lib as L
from oracle import sh_oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = {"fp64": 1e-10, "fp32": 1e-5}
ETOL = {"fp64": 1e-10, "fp32": 5e-6}


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def oracle_params(p: S.Params) -> O.Params:
    return O.Params(n=p.n, dx=p.dx, dt=p.dt, eps=p.eps, beta=p.beta, gamma=p.gamma, alpha=p.alpha, q0=p.q0,
                    eta=p.eta, rho=p.rho, nonlinearity=p.nonlinearity, scheme=p.scheme, w_mid=p.w_mid)


def golden(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    kw = {k[6:]: d[k].item() for k in d.files if k.startswith("param_")}
    kw.pop("sub_sigma", None)
    kw.pop("sub_z0", None)
    return d, kw


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("name,boundary", [
    ("periodic_plain_16", "periodic"),
    ("periodic_lamellae_32", "periodic"),
    ("periodic_imex_quadcubic_16", "periodic"),
    ("periodic_penalty_16", "periodic"),
    ("neumann_hyperboloid_16", "neumann"),
    ("neumann_l1_32", "neumann"),
])
def test_golden_vectors(name, boundary, prec):
    d, kw = golden(name)
    p = S.Params(boundary=boundary, precision=prec, **{k: v for k, v in kw.items() if k in S.Params.__dataclass_fields__})
    if "l1" in d.files:
        p.l1_interval = int(d["steps"])
    with S.Solver(p) as s:
        s.set_psi(d["psi0"])
        s.step(int(d["steps"]))
        psi = s.get_psi()
        assert rel(psi, d["psi"]) <= TOL[prec]
        if "energy" in d.files:
            e = s.energy()[0]
            assert abs(e - float(d["energy"])) <= ETOL[prec] * abs(float(d["energy"]))
        if "l1" in d.files:
            l1, cnt = s.l1()
            assert cnt == 1
            assert abs(l1[0] - float(d["l1"])) <= (1e-9 if prec == "fp64" else 1e-3) * abs(float(d["l1"]))


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("boundary", ["periodic", "neumann"])
@pytest.mark.parametrize("n", [32, 64, 128])
def test_live_oracle_100_steps(n, boundary, prec):
    p = S.Params(n=n, boundary=boundary, precision=prec, dt=0.05, eps=-0.7)
    psi0 = 1.3 * np.cos(np.arange(n) * p.dx)[None, None, :] + S.ic.noise(n, 7, 0.2)
    orc = (O.PeriodicOracle if boundary == "periodic" else O.NeumannOracle)(psi0, oracle_params(p))
    orc.run(100)
    with S.Solver(p) as s:
        s.set_psi(psi0)
        s.step(100)
        assert rel(s.get_psi(), orc.psi) <= TOL[prec]
        efun = O.energy_spectral_periodic if boundary == "periodic" else O.energy_spectral_neumann
        eo = efun(orc.psi, oracle_params(p))
        assert abs(s.energy()[0] - eo) <= ETOL[prec] * abs(eo)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("boundary", ["periodic", "neumann"])
def test_live_oracle_256_baseline_ics(boundary, prec):
    """The 256^3 workloads' own initial conditions, a few steps against the oracle."""
    n = 256
    p = S.Params(n=n, boundary=boundary, precision=prec, dt=0.05)
    psi0 = S.ic.noise(n, 0) if boundary == "periodic" else S.ic.hyperboloid(n, p.dx, seed=0)
    orc = (O.PeriodicOracle if boundary == "periodic" else O.NeumannOracle)(psi0, oracle_params(p))
    orc.run(4)
    with S.Solver(p) as s:
        s.set_psi(psi0)
        s.step(4)
        assert rel(s.get_psi(), orc.psi) <= TOL[prec]


@pytest.mark.parametrize("boundary", ["periodic", "neumann"])
@pytest.mark.parametrize("n,prec", [(16, "fp64"), (256, "fp64"), (256, "fp32"), (512, "fp32")])
def test_linear_growth_factor_full_size(n, prec, boundary):
    """beta = gamma = 0: every step multiplies a grid mode by (1+dt a/2)/(1-dt a/2)."""
    p = S.Params(n=n, boundary=boundary, precision=prec, dt=0.1, eps=0.1, beta=0.0, gamma=0.0)
    z = np.arange(n)
    m = n // 8 + 1
    if boundary == "periodic":
        q = 2 * math.pi * m / (n * p.dx)
        prof = np.cos(2 * math.pi * m * z / n)
    else:
        q = math.pi * m / (n * p.dx)
        prof = np.cos(math.pi * m * (z + 0.5) / n)
    psi0 = 1e-3 * np.broadcast_to(prof[None, :, None] * np.ones((1, 1, n)), (n, n, n)).copy()
    a = p.eps - (q * q - 1.0) ** 2
    g = (1 + p.dt * a / 2) / (1 - p.dt * a / 2)
    with S.Solver(p) as s:
        s.set_psi(psi0)
        s.step(3)
        assert rel(s.get_psi(), g ** 3 * psi0) <= (1e-12 if prec == "fp64" else 1e-6)


def test_fp64_512_reports_unsupported():
    """512^3 in FP64 needs more shared memory per CTA than the plane pass can use."""
    with pytest.raises(S.ShError) as e:
        S.Solver(S.Params(n=512, precision="fp64"))
    assert e.value.code == L.SH_EUNSUPPORTED


@pytest.mark.parametrize("boundary", ["periodic", "neumann"])
def test_fp32_matches_fp64_at_256(boundary):
    n = 256
    psi0 = S.ic.undulated_lamellae(n, 2 * math.pi / 8, amp=1.3, seed=1) + S.ic.noise(n, 2, 0.05)
    out = {}
    for prec in ("fp64", "fp32"):
        with S.Solver(S.Params(n=n, boundary=boundary, precision=prec, eps=-0.7)) as s:
            s.set_psi(psi0)
            s.step(100)
            out[prec] = s.get_psi()
    assert rel(out["fp32"], out["fp64"]) <= 1e-5


@pytest.mark.parametrize("boundary", ["periodic", "neumann"])
def test_energy_trace_and_lyapunov(boundary):
    n = 32
    p = S.Params(n=n, boundary=boundary, precision="fp64", dt=0.02, eps=-0.7, energy_trace=True)
    psi0 = 1.3 * np.cos(np.arange(n) * p.dx)[None, None, :] + S.ic.noise(n, 9, 0.3)
    orc = (O.PeriodicOracle if boundary == "periodic" else O.NeumannOracle)(psi0, oracle_params(p))
    efun = O.energy_spectral_periodic if boundary == "periodic" else O.energy_spectral_neumann
    ref = []
    for _ in range(20):
        orc.step()
        ref.append(efun(orc.psi, oracle_params(p)))
    with S.Solver(p) as s:
        s.set_psi(psi0)
        s.step(12)
        s.step(8)
        tr = s.energy_trace()[:, 0]
    assert tr.shape == (20,)
    assert np.allclose(tr, ref, rtol=1e-10, atol=0)
    assert (np.diff(tr) <= 1e-9 * np.abs(tr[:-1])).all()


@pytest.mark.parametrize("boundary", ["periodic", "neumann"])
def test_l1_monitor_matches_oracle(boundary):
    n = 32
    p = S.Params(n=n, boundary=boundary, precision="fp64", eps=-0.7, l1_interval=5)
    psi0 = 1.3 * np.cos(np.arange(n) * p.dx)[None, None, :] + S.ic.noise(n, 10, 0.3)
    orc = (O.PeriodicOracle if boundary == "periodic" else O.NeumannOracle)(psi0, oracle_params(p))
    with S.Solver(p) as s:
        s.set_psi(psi0)
        for k in range(3):
            for _ in range(5):
                prev = orc.psi.copy()
                orc.step()
            s.step(5)
            l1, cnt = s.l1()
            assert cnt == k + 1
            assert abs(l1[0] - O.l1_monitor(orc.psi, prev, p.dt)) <= 1e-10 * O.l1_monitor(orc.psi, prev, p.dt)


def test_l1_every_step():
    n = 16
    p = S.Params(n=n, precision="fp64", l1_interval=1)
    psi0 = S.ic.noise(n, 11, 0.5)
    orc = O.PeriodicOracle(psi0, oracle_params(p))
    orc.step()
    with S.Solver(p) as s:
        s.set_psi(psi0)
        s.step(1)
        l1, cnt = s.l1()
    assert cnt == 1 and abs(l1[0] - O.l1_monitor(orc.psi, psi0, p.dt)) <= 1e-10 * l1[0]


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_batched_replicas_are_independent(prec):
    n, b = 64, 4
    eps = np.linspace(-0.9, -0.5, b)
    psi0 = S.ic.noise_batch(n, range(b))
    p = S.Params(n=n, batch=b, precision=prec, eps_per_replica=tuple(eps))
    with S.Solver(p) as s:
        s.set_psi(psi0)
        s.step(30)
        allpsi = s.get_psi()
        eb = s.energy()
    for r in range(b):
        orc = O.PeriodicOracle(psi0[r], oracle_params(S.Params(n=n, eps=eps[r])))
        orc.run(30)
        assert rel(allpsi[r], orc.psi) <= TOL[prec]
        eo = O.energy_spectral_periodic(orc.psi, oracle_params(S.Params(n=n, eps=eps[r])))
        assert abs(eb[r] - eo) <= ETOL[prec] * abs(eo)


@pytest.mark.parametrize("boundary", ["periodic", "neumann"])
def test_checkpoint_roundtrip_is_bit_exact(boundary):
    n = 32
    p = S.Params(n=n, boundary=boundary, precision="fp64")
    with S.Solver(p) as s:
        s.set_psi(S.ic.noise(n, 12, 0.4))
        s.step(7)
        blob = s.checkpoint()
        s.step(9)
        a = s.get_psi()
        s.restore(blob)
        assert s.steps_taken == 7
        s.step(9)
        b = s.get_psi()
    assert np.array_equal(a, b)


def test_padded_layout_roundtrip():
    n = 32
    p = S.Params(n=n, precision="fp64")
    psi0 = S.ic.noise(n, 13)
    padded = np.zeros((n, n, 2 * (n // 2 + 1)))
    padded[:, :, :n] = psi0
    with S.Solver(p) as s:
        s.set_psi(padded, layout=L.SH_LAYOUT_PADDED)
        assert np.array_equal(s.get_psi(), psi0)
        back = s.get_psi(layout=L.SH_LAYOUT_PADDED)
    assert np.array_equal(back[:, :, :n], psi0)


def test_nonfinite_state_is_reported():
    n = 16
    psi0 = S.ic.noise(n, 14)
    psi0[3, 4, 5] = np.nan
    with S.Solver(S.Params(n=n)) as s:
        s.set_psi(psi0)
        with pytest.raises(S.ShError) as e:
            s.step(1)
        assert e.value.code == L.SH_ENONFINITE


def test_state_errors():
    with S.Solver(S.Params(n=16)) as s:
        with pytest.raises(S.ShError) as e:
            s.step(1)
        assert e.value.code == L.SH_ESTATE


def test_run_host_roundtrip_matches_steps():
    n = 32
    psi0 = S.ic.noise(n, 15)
    p = S.Params(n=n, precision="fp32")
    with S.Solver(p) as s:
        a = s.run(psi0, 10)
        s.set_psi(psi0)
        s.step(10)
        b = s.get_psi()
    assert np.array_equal(a, b)
