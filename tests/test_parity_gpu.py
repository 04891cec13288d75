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
    return d, kw


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("name,boundary", [
    ("periodic_plain_16", "periodic"),
    ("periodic_lamellae_32", "periodic"),
    ("periodic_imex_quadcubic_16", "periodic"),
    ("periodic_penalty_16", "periodic"),
    ("neumann_hyperboloid_16", "neumann"),
    ("neumann_l1_32", "neumann"),
    ("periodic_advected_16", "periodic"),
    ("neumann_substrate_16", "neumann"),
])
def test_golden_vectors(name, boundary, prec):
    d, kw = golden(name)
    p = S.Params(boundary=boundary, precision=prec, **{k: v for k, v in kw.items() if k in S.Params.__dataclass_fields__})
    p.advection = bool(d["advect"]) if "advect" in d.files else False
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


def _golden64_ic(kind, n, dx):
    if kind == "noise11+lamellae1.3":
        return S.ic.noise(n, 11, 0.2) + 1.3 * np.cos(np.arange(n) * dx)[None, None, :]
    if kind == "hyperboloid12":
        return S.ic.hyperboloid(n, dx, r0_cells=12.0, seed=12)
    raise ValueError(kind)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("name,boundary", [("periodic_plain_64", "periodic"), ("neumann_hyperboloid_64", "neumann")])
def test_golden_vectors_64(name, boundary, prec):
    """64^3 golden states, stored compactly (every 4th point per axis and two global sums);
    the seeded initial condition is regenerated here."""
    d, kw = golden(name)
    p = S.Params(boundary=boundary, precision=prec, **{k: v for k, v in kw.items() if k in S.Params.__dataclass_fields__})
    with S.Solver(p) as s:
        s.set_psi(_golden64_ic(str(d["ic_kind"]), p.n, p.dx))
        s.step(int(d["steps"]))
        psi = s.get_psi()
    assert rel(psi[::4, ::4, ::4], d["psi_sub"]) <= TOL[prec]
    assert abs(float(np.sum(psi * psi)) - float(d["sum_sq"])) <= TOL[prec] * float(d["sum_sq"])
    assert abs(float(np.sum(np.abs(psi))) - float(d["sum_abs"])) <= TOL[prec] * float(d["sum_abs"])


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
def test_live_oracle_256_workload_ics(boundary, prec):
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
@pytest.mark.parametrize("n,prec", [(16, "fp64"), (256, "fp64"), (256, "fp32"), (512, "fp32"), (512, "fp64")])
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


@pytest.mark.parametrize("n,prec", [(256, "fp32"), (512, "fp64")])
def test_advected_single_mode_is_the_plain_growth(n, prec):
    """Known answer for the advected step at full size (512^3 FP64 runs its plane
    passes with direct exchanges): for psi = A cos(q z) the stress
    S = (L psi) grad psi = -(1/2) opSH q A^2 sin(2 q z) e_z is a gradient, the
    projector removes it, u = 0, and with beta = gamma = 0 every step multiplies
    the mode by (1 + dt a/2)/(1 - dt a/2)."""
    p = S.Params(n=n, precision=prec, dt=0.1, eps=0.1, beta=0.0, gamma=0.0, advection=True)
    m = n // 8 + 1
    q = 2 * math.pi * m / (n * p.dx)
    psi0 = 1e-3 * np.broadcast_to(np.cos(2 * math.pi * m * np.arange(n) / n)[None, None, :], (n, n, n)).copy()
    a = p.eps - (q * q - 1.0) ** 2
    g = (1 + p.dt * a / 2) / (1 - p.dt * a / 2)
    with S.Solver(p) as s:
        s.set_psi(psi0)
        s.step(3)
        assert rel(s.get_psi(), g ** 3 * psi0) <= (1e-12 if prec == "fp64" else 1e-6)
        u = s.velocity()
    # the velocity the projector removed, |S| / (rho eta q^2) with S = (1/2) opSH q A^2,
    # is left at the level of the transforms' rounding (FP32: the rounding noise of
    # L psi grows with opSH at large |k|)
    removed = 0.5 * (q * q - 1.0) ** 2 * q * 1e-6 / (q * q)
    assert max(np.abs(c).max() for c in u) <= (1e-10 if prec == "fp64" else 1e-2) * removed


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


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("boundary", ["periodic", "neumann"])
def test_replica_blocks_are_bit_exact(boundary, prec):
    """replica_block: blocks of replicas take 16 steps at a time while their state
    stays in L2; every replica's result is bit for bit the unblocked one, and
    replica 0 matches the oracle."""
    n, b = 64, 11
    eps = np.linspace(-0.9, -0.5, b)
    psi0 = S.ic.noise_batch(n, range(b), 0.3) + 1.3 * np.cos(np.arange(n) * 2 * math.pi / 8)[None, None, None, :]
    out = {}
    for blk in (0, 4):
        p = S.Params(n=n, batch=b, boundary=boundary, precision=prec, eps_per_replica=tuple(eps), replica_block=blk)
        with S.Solver(p) as s:
            s.set_psi(psi0)
            s.step(40)  # two replayed 16-step blocks and 8 direct steps
            out[blk] = s.get_psi()
    assert np.array_equal(out[0], out[4])
    q = S.Params(n=n, boundary=boundary, eps=eps[0])
    orc = (O.PeriodicOracle if boundary == "periodic" else O.NeumannOracle)(psi0[0], oracle_params(q))
    orc.run(40)
    assert rel(out[4][0], orc.psi) <= TOL[prec]


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


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("n", [16, 32, 64, 128])
def test_advected_matches_oracle(n, prec):
    """Periodic step with the Fourier Stokes advection (periodicFFT/pf3d.cpp:395-485)."""
    p = S.Params(n=n, advection=True, precision=prec, dt=0.01, eps=-0.7, eta=1.0, rho=1.0)
    psi0 = S.ic.pf3d_lamellae(n, p.dx, kmin=1, kmax=n - 1) + S.ic.noise(n, 21, 0.05)
    orc = O.PeriodicOracle(psi0, oracle_params(p), advect=True)
    steps = 20 if n <= 64 else 5
    orc.run(steps)
    with S.Solver(p) as s:
        s.set_psi(psi0)
        s.step(steps)
        assert rel(s.get_psi(), orc.psi) <= TOL[prec]
        eo = O.energy_spectral_periodic(orc.psi, oracle_params(p))
        assert abs(s.energy()[0] - eo) <= ETOL[prec] * abs(eo)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_advected_256_undulated_lamellae(prec):
    """The advected 256^3 workload's own IC, a few steps against the oracle."""
    n = 256
    p = S.Params(n=n, advection=True, precision=prec, dt=0.02)
    psi0 = S.ic.undulated_lamellae(n, p.dx, seed=0)
    orc = O.PeriodicOracle(psi0, oracle_params(p), advect=True)
    orc.run(2)
    with S.Solver(p) as s:
        s.set_psi(psi0)
        s.step(2)
        assert rel(s.get_psi(), orc.psi) <= TOL[prec]


def test_advected_checkpoint_roundtrip():
    n = 32
    p = S.Params(n=n, advection=True, precision="fp64", dt=0.01)
    with S.Solver(p) as s:
        s.set_psi(S.ic.noise(n, 22, 0.5))
        s.step(3)
        blob = s.checkpoint()
        s.step(4)
        a = s.get_psi()
        s.restore(blob)
        s.step(4)
        b = s.get_psi()
    assert np.array_equal(a, b)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("n", [32, 64])
def test_surface_step_matches_oracle(n, prec):
    """surfTrack (periodicFFT/surfTrack.cpp:592-626, 767-806): crossing z of the new
    psi per column, with v_n, H and K from the fields of the step."""
    p = S.Params(n=n, advection=True, precision=prec, dt=0.02, eps=-0.7)
    # lamellae undulated along x and y, so that both curvatures are non-zero
    c = np.arange(n) * p.dx
    lam = n / 2 * p.dx
    # (off-grid phases: no exact zeros of psi on grid points, whose sign rounding would decide)
    h = 0.83 * p.dx * (np.sin(2 * np.pi * c / lam + 0.3)[:, None, None] + np.cos(2 * np.pi * c / lam + 0.7)[None, :, None])
    psi0 = 1.3 * np.cos(c[None, None, :] - h - 0.37)
    orc = O.PeriodicOracle(psi0, oracle_params(p), advect=True)
    orc.run(3)
    orc.step()
    zo, vo, ho, ko = O.surface_scan(orc.psi, *orc.surface_fields())
    with S.Solver(p) as s:
        s.set_psi(psi0)
        s.step(3)
        z, vn, hh, kk = s.surface_step()
        assert rel(s.get_psi(), orc.psi) <= TOL[prec]
    found = zo >= 0
    assert found.mean() > 0.9
    same = z == zo
    assert same.mean() >= (1.0 if prec == "fp64" else 0.99)
    m = same & found
    # FP32: d_t psi = eps psi - L psi + N cancels O(1) terms down to O(0.05)
    tol = 1e-8 if prec == "fp64" else 1e-3
    for got, ref in ((vn, vo), (hh, ho), (kk, ko)):
        scale = max(np.abs(ref[m]).max(), 1e-3)
        assert np.abs(got[m] - ref[m]).max() <= tol * scale
    assert np.abs(ko[m]).max() > 1e-4  # the IC really is doubly curved
    assert np.isnan(vn[~(z >= 0)]).all()


def test_surface_step_needs_advection():
    with S.Solver(S.Params(n=16)) as s:
        s.set_psi(S.ic.noise(16, 1))
        with pytest.raises(S.ShError) as e:
            s.surface_step()
        assert e.value.code == L.SH_EINVAL


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("n,steps,k", [(16, 10, 4), (32, 12, 5), (32, 7, 50)])
def test_adjoint_matches_oracle(n, steps, k, prec):
    """Discrete adjoint of CNAB2 (checkpoints every k steps) against the FP64 oracle
    adjoint, for L = 1/2 ||psi_T - target||^2 with a lamellar target 0.5 cos(1.05 z)."""
    p = S.Params(n=n, precision=prec, dt=0.05)
    psi0 = S.ic.noise(n, 31, 0.1) + 1.2 * np.cos(np.arange(n) * p.dx)[None, None, :]
    target = 0.5 * np.broadcast_to(np.cos(1.05 * np.arange(n) * p.dx)[None, None, :], (n, n, n))
    loss, ge, gq, gpsi = O.adjoint_gradients_periodic(psi0, oracle_params(p), steps, target)
    orc = O.PeriodicOracle(psi0, oracle_params(p))
    orc.run(steps)
    with S.Solver(p) as s:
        s.set_psi(psi0)
        s.step(steps)
        psi_t = s.get_psi()
        g_e, g_q, g_p = s.adjoint(psi0, steps, psi_t - target, ckpt_every=k)
    tol = 1e-9 if prec == "fp64" else 1e-4
    assert abs(g_e[0] - ge) <= tol * abs(ge)
    assert abs(g_q[0] - gq) <= tol * abs(gq)
    assert rel(g_p, gpsi) <= tol


def test_adjoint_finite_differences_fp32_forward():
    """FP32 forward + FP64 gradient accumulation against central differences of the
    FP64 oracle loss (h = 1e-4), as the differentiation workload asks."""
    import dataclasses
    n, steps = 16, 20
    p = S.Params(n=n, precision="fp32", dt=0.05)
    psi0 = S.ic.noise(n, 32, 0.1) + 1.2 * np.cos(np.arange(n) * p.dx)[None, None, :]
    target = 0.5 * np.broadcast_to(np.cos(1.05 * np.arange(n) * p.dx)[None, None, :], (n, n, n))
    op = oracle_params(p)

    def lossf(pp):
        o = O.PeriodicOracle(psi0, pp)
        o.run(steps)
        return 0.5 * ((o.psi - target) ** 2).sum()

    h = 1e-4
    fe = (lossf(dataclasses.replace(op, eps=op.eps + h)) - lossf(dataclasses.replace(op, eps=op.eps - h))) / (2 * h)
    fq = (lossf(dataclasses.replace(op, q0=op.q0 + h)) - lossf(dataclasses.replace(op, q0=op.q0 - h))) / (2 * h)
    orc = O.PeriodicOracle(psi0, op)
    orc.run(steps)
    with S.Solver(p) as s:
        g_e, g_q, _ = s.adjoint(psi0, steps, orc.psi - target, ckpt_every=5)
    assert abs(g_e[0] - fe) <= 1e-4 * abs(fe)
    assert abs(g_q[0] - fq) <= 1e-4 * abs(fq)


def test_adjoint_batched_replicas():
    n, steps, b = 16, 8, 3
    eps = (-0.9, -0.7, -0.5)
    p = S.Params(n=n, batch=b, precision="fp64", eps_per_replica=eps)
    psi0 = S.ic.noise_batch(n, (40, 41, 42), 0.3)
    lam = S.ic.noise_batch(n, (43, 44, 45), 1.0)
    with S.Solver(p) as s:
        g_e, g_q, g_p = s.adjoint(psi0, steps, lam, ckpt_every=3)
    for r in range(b):
        with S.Solver(S.Params(n=n, precision="fp64", eps=eps[r])) as s1:
            e1, q1, p1 = s1.adjoint(psi0[r], steps, lam[r], ckpt_every=8)
        assert abs(g_e[r] - e1[0]) <= 1e-10 * abs(e1[0])
        assert abs(g_q[r] - q1[0]) <= 1e-10 * abs(q1[0])
        assert rel(g_p[r], p1) <= 1e-10


def test_graph_replay_matches_direct_launches():
    """Steps replayed from the captured CUDA graph equal steps launched one by one."""
    n = 64
    psi0 = S.ic.noise(n, 50)
    with S.Solver(S.Params(n=n, precision="fp32")) as a, S.Solver(S.Params(n=n, precision="fp32", l1_interval=1000)) as b:
        a.set_psi(psi0)
        b.set_psi(psi0)
        a.step(40)          # 2 graph chunks of 16 + 8 direct steps
        b.step(40)          # L1 bookkeeping forces direct launches
        assert a.steps_taken == b.steps_taken == 40
        assert np.array_equal(a.get_psi(), b.get_psi())
        assert a.kernel_launches == b.kernel_launches


def test_autotune_picks_a_built_variant(tmp_path, monkeypatch):
    from smectic3d_b200 import autotune
    monkeypatch.setenv("SMECTIC_B200_CACHE", str(tmp_path / "tuned.json"))
    p = S.Params(n=64, batch=8, precision="fp32")
    rec = autotune.tune(p, steps=5)
    assert rec["variant"] in autotune.CANDIDATES[64]
    assert (tmp_path / "tuned.json").exists()
    with S.Solver(S.Params(n=64, batch=8, precision="fp32", variant=-1)) as s:
        assert s.params.variant == rec["variant"]
