"""Pins of the FP64 oracle (CPU only).

The reference ships no tests or golden outputs and cannot be built here, so the
oracle is pinned to analytic known-answer tests of the reference's algorithm:
FFTW's transform conventions, the exact CNAB2 growth factor of grid modes
(the pf3dVal validation, periodicFFT/pf3dVal.cpp:214-331, restricted to
grid-commensurate wavenumbers), the lamellar amplitude of the reference ICs,
Lyapunov decrease, the Stokes projector and the surfTrack crossing.
"""
import dataclasses
import math

import numpy as np
import pytest
import scipy.fft as sfft

from oracle import sh_oracle as O


def test_wavenumbers_follow_reference_formula():
    n, dx = 16, 2 * math.pi / 8
    q = O.kvec_periodic(n, dx)
    # periodicFFT/pf3d.cpp:176-182 (Vqy form, explicit Nyquist +pi/dy)
    ref = np.zeros(n)
    ref[n // 2] = math.pi / dx
    for j in range(1, n // 2):
        ref[j] = 2 * math.pi * j / (dx * n)
        ref[n // 2 + j] = -(n // 2 - j) * 2 * math.pi / (dx * n)
    assert np.allclose(q, ref, rtol=0, atol=1e-15)
    qd = O.kvec_dct(n, dx)
    assert np.allclose(qd, math.pi * np.arange(n) / (dx * n))


def test_fftw_scale_conventions():
    rng = np.random.default_rng(0)
    a = rng.standard_normal((8, 8, 8))
    # unnormalised r2c then c2r multiplies by N^3 (the reference scales by 1/NG)
    assert np.allclose(O.c2r(O.r2c(a), 8), a * 512, atol=1e-10)
    # REDFT10 then REDFT01 multiplies by (2N)^3 (cosNoAdvMorph scale 0.125/N^3)
    assert np.allclose(O.idct3d(O.dct3d(a)), a * 8 * 512, atol=1e-9)
    # REDFT10 definition: Y[k] = 2 sum x[n] cos(pi (2n+1) k / 2N)
    x = rng.standard_normal(8)
    k = np.arange(8)[:, None]
    nn = np.arange(8)[None, :]
    y = 2 * (x[None, :] * np.cos(np.pi * (2 * nn + 1) * k / 16)).sum(1)
    assert np.allclose(sfft.dct(x, type=2), y)
    # REDFT01: Y[n] = X[0] + 2 sum_{k>0} X[k] cos(pi k (2n+1) / 2N)
    y3 = x[0] + 2 * (x[None, 1:] * np.cos(np.pi * np.arange(1, 8)[None, :] * (2 * np.arange(8)[:, None] + 1) / 16)).sum(1)
    assert np.allclose(sfft.dct(x, type=3), y3)


def test_c2r_semantics_non_hermitian():
    """FFTW c2r: complex inverse over x, y, then the real part on kz=0, N/2."""
    rng = np.random.default_rng(1)
    n = 8
    a = rng.standard_normal((n, n, n // 2 + 1)) + 1j * rng.standard_normal((n, n, n // 2 + 1))
    g = np.fft.ifft(np.fft.ifft(a, axis=0), axis=1) * n * n
    full = np.zeros((n, n, n), complex)
    full[:, :, : n // 2 + 1] = g
    full[:, :, 0] = g[:, :, 0].real
    full[:, :, n // 2] = g[:, :, n // 2].real
    for kz in range(n // 2 + 1, n):
        full[:, :, kz] = np.conj(g[:, :, n - kz])
    ref = np.fft.ifft(full, axis=2).real * n
    assert np.allclose(O.c2r(a, n), ref, atol=1e-12)


@pytest.mark.parametrize("boundary", ["periodic", "neumann"])
def test_linear_growth_factor_kat(boundary):
    """beta = gamma = 0: one CNAB2 step multiplies mode q by (1+dt a/2)/(1-dt a/2),
    a = eps - (q^2 - q0^2)^2 -- the pf3dVal validation on grid modes."""
    n = 32
    p = O.Params(n=n, dt=0.1, eps=0.1, beta=0.0, gamma=0.0)
    kv = O.kvec_periodic(n, p.dx) if boundary == "periodic" else O.kvec_dct(n, p.dx)
    z = np.arange(n)
    for m in (1, 3, 4, 5, 8):
        q = kv[m]
        if boundary == "periodic":
            prof = np.cos(2 * math.pi * m * z / n)
        else:
            prof = np.cos(math.pi * m * (z + 0.5) / n)
        psi0 = 1e-4 * np.broadcast_to(prof, (n, n, n)).copy()
        orc = (O.PeriodicOracle if boundary == "periodic" else O.NeumannOracle)(psi0, p)
        a = p.eps - (q * q - p.q0 ** 2) ** 2
        g = (1 + p.dt * a / 2) / (1 - p.dt * a / 2)
        for s in range(1, 4):
            orc.step()
            assert np.allclose(orc.psi, g ** s * psi0, rtol=1e-11, atol=1e-18)


def test_lamellar_amplitude_matches_reference_ic():
    """psi = A cos(q0 z) at eps=-0.7 relaxes to the reference amplitude 1.328
    (cosFFT/comet/cosNoAdvMorph.cpp:322); one-mode estimate 1.3288."""
    n = 16
    p = O.Params(n=n, dt=0.1, eps=-0.7)
    z = np.arange(n) * p.dx
    psi0 = np.broadcast_to(1.0 * np.cos(z), (n, n, n)).copy()
    orc = O.PeriodicOracle(psi0, p)
    orc.run(600)
    amp = orc.psi.max()
    assert abs(amp - 1.328) < 0.03
    psi0 = np.broadcast_to(0.5 * np.cos(z), (n, n, n)).copy()  # below threshold decays
    orc = O.PeriodicOracle(psi0, p)
    orc.run(300)
    assert np.abs(orc.psi).max() < 0.05


@pytest.mark.parametrize("boundary", ["periodic", "neumann"])
def test_lyapunov_decrease(boundary):
    n = 16
    p = O.Params(n=n, dt=0.02, eps=-0.7)
    psi0 = 1.3 * np.cos(np.arange(n) * p.dx)[None, None, :] + np.random.default_rng(2).uniform(-0.3, 0.3, (n, n, n))
    orc = (O.PeriodicOracle if boundary == "periodic" else O.NeumannOracle)(psi0, p)
    efun = O.energy_spectral_periodic if boundary == "periodic" else O.energy_spectral_neumann
    e = [efun(orc.psi, p)]
    for _ in range(40):
        orc.step()
        e.append(efun(orc.psi, p))
    assert all(e[i + 1] <= e[i] + 1e-9 * abs(e[i]) for i in range(len(e) - 1))


def test_energy_forms_agree_on_smooth_field():
    """FD+trapz (energyPsi.m) and spectral forms agree as the grid resolves psi."""
    n = 64
    p = O.Params(n=n, dx=2 * math.pi / 32, eps=-0.7)
    z = np.arange(n) * p.dx
    psi = np.broadcast_to(1.3 * np.cos(z), (n, n, n)).copy()
    es = O.energy_spectral_periodic(psi, p)
    ef = O.energy_fd_trapz(psi, p)
    # trapz drops half of the two end planes of a periodic sum; FD Laplacian O(dx^2)
    assert abs(es - ef) / abs(es) < 0.05


def test_stokes_projector_identities():
    n = 16
    p = O.Params(n=n)
    rng = np.random.default_rng(3)
    psi = rng.uniform(-1, 1, (n, n, n))
    orc = O.PeriodicOracle(psi, p, advect=True)
    (ux, uy, uz), grads, lpsi = orc.velocity(O.r2c(psi))
    uq = [O.r2c(u) for u in (ux, uy, uz)]
    div = orc.qx * uq[0] + orc.qy * uq[1] + orc.qz * uq[2]
    # q . u = 0 away from the Nyquist planes (where q_{N/2} = +pi/dx breaks the
    # Hermitian pairing of the C2R/R2C round trip)
    inner = div[1:n // 2, 1:n // 2, 1:n // 2]
    assert np.abs(inner).max() < 1e-9 * max(1.0, np.abs(uq[0]).max())
    assert abs(uq[0][0, 0, 0]) < 1e-12 and abs(uq[2][0, 0, 0]) < 1e-12
    # single-mode forcing: u = S_perp / (rho eta q^2)
    s = np.zeros((n, n, n))
    x = np.arange(n) * p.dx
    s = np.broadcast_to(np.cos(2 * math.pi * 2 * x / (n * p.dx))[None, None, :], (n, n, n)).copy()
    sq = O.r2c(s)
    zero = np.zeros_like(sq)
    dot = orc.qx * zero + orc.qy * sq + orc.qz * zero
    uy = O.c2r(orc.scale * orc.cm1 * (sq - orc.cm2y * dot), n)
    # forcing along y varying along z is transverse: u_y = S / q^2
    q = 2 * math.pi * 2 / (n * p.dx)
    assert np.allclose(uy, s / q ** 2, atol=1e-12)


def test_surface_scan_planar_front():
    """psi = cos(q0 (z - z0)) + tilt-free: the crossing sits at the first
    descending zero after psi > 0.1, H = K = 0."""
    n = 32
    p = O.Params(n=n, dt=0.01, beta=0.0, gamma=0.0, eps=0.0)
    z = np.arange(n) * p.dx
    psi0 = np.broadcast_to(np.cos(z - 0.3), (n, n, n)).copy()
    orc = O.PeriodicOracle(psi0, p)
    orc.step()
    fields = orc.surface_fields()
    zi, vn, hh, kk = O.surface_scan(orc.psi, *fields)
    col = orc.psi[0, 0]
    k = next(k for k in range(1, n) if col[k] < 0 and any(col[:k] > 0.1))
    assert (zi == k).all()
    assert np.abs(hh).max() < 1e-10 and np.abs(kk).max() < 1e-10
    assert np.isfinite(vn).all()


@pytest.mark.parametrize("n", [16, 32])
def test_surface_scan_vectorised_equals_column_loop(n):
    """The whole-array scan used for the 256^3 fixtures equals the per-column
    restatement of surfTrack.cpp:767-806 on doubly curved lamellae."""
    p = O.Params(n=n, dt=0.02, eps=-0.7)
    c = np.arange(n) * p.dx
    lam = n / 2 * p.dx
    h = 0.83 * p.dx * (np.sin(2 * np.pi * c / lam + 0.3)[:, None, None] + np.cos(2 * np.pi * c / lam + 0.7)[None, :, None])
    orc = O.PeriodicOracle(1.3 * np.cos(c[None, None, :] - h - 0.37), p, advect=True)
    orc.run(2)
    orc.step()
    f = orc.surface_fields()
    for a, b in zip(O.surface_scan(orc.psi, *f), O.surface_scan_vec(orc.psi, *f)):
        assert np.array_equal(a, b, equal_nan=True)


def test_dominant_wavenumber_of_single_modes():
    """A single grid mode puts all its power in its own shell, in both boxes."""
    n, dx = 32, 2 * math.pi / 8
    i = np.arange(n)
    for m in (3, 5):
        per = np.cos(2 * math.pi * m * i / n)[None, None, :] * np.cos(2 * math.pi * 2 * i / n)[:, None, None]
        assert math.isclose(O.dominant_wavenumber(np.broadcast_to(per, (n, n, n)), dx),
                            round(math.hypot(m, 2)) * 2 * math.pi / (n * dx))
        neu = np.cos(math.pi * m * (i + 0.5) / n)[None, None, :] * np.cos(math.pi * 4 * (i + 0.5) / n)[None, :, None]
        assert math.isclose(O.dominant_wavenumber_neumann(np.broadcast_to(neu, (n, n, n)), dx),
                            round(math.hypot(m, 4)) * math.pi / (n * dx))


def test_adjoint_matches_finite_differences():
    n = 8
    p = O.Params(n=n, dt=0.05)
    rng = np.random.default_rng(4)
    psi0 = rng.uniform(-1.2, 1.2, (n, n, n))
    tgt = 0.5 * np.broadcast_to(np.cos(1.05 * np.arange(n) * p.dx), (n, n, n))
    steps = 6
    loss, ge, gq, gpsi = O.adjoint_gradients_periodic(psi0, p, steps, tgt)

    def lossf(pp, ps):
        o = O.PeriodicOracle(ps, pp)
        o.run(steps)
        return 0.5 * ((o.psi - tgt) ** 2).sum()

    h = 1e-5
    fe = (lossf(dataclasses.replace(p, eps=p.eps + h), psi0) - lossf(dataclasses.replace(p, eps=p.eps - h), psi0)) / (2 * h)
    fq = (lossf(dataclasses.replace(p, q0=p.q0 + h), psi0) - lossf(dataclasses.replace(p, q0=p.q0 - h), psi0)) / (2 * h)
    d = np.zeros_like(psi0)
    d[1, 2, 3] = 1
    fp = (lossf(p, psi0 + h * d) - lossf(p, psi0 - h * d)) / (2 * h)
    assert abs(ge - fe) <= 1e-6 * max(1, abs(fe))
    assert abs(gq - fq) <= 1e-6 * max(1, abs(fq))
    assert abs(gpsi[1, 2, 3] - fp) <= 1e-6 * max(1, abs(fp))


def test_golden_fixtures_reproduce():
    """The committed golden vectors (tests/golden) are what the oracle computes."""
    from tests.golden import make_golden as G
    for name, fn in G.CASES.items():
        ref = np.load(G.path(name))
        got = fn()
        for k in ref.files:
            if ref[k].dtype.kind in "fc":
                assert np.allclose(got[k], ref[k], rtol=1e-12, atol=1e-14), (name, k)
            else:
                assert (np.asarray(got[k]) == ref[k]).all(), (name, k)


def test_curvature_pass_sphere_kat():
    """Neumann curvature pass (cosNoAdvMorphCurv.cpp:874-965) on spherical level
    sets psi = cos(r - R): Megrabov's H = 2/r and K = 1/r^2 at the crossing,
    to the accuracy of the difference gradients (dx = 2 pi / 32)."""
    n = 48
    dx = 2 * math.pi / 32
    p = O.Params(n=n, dx=dx, dt=0.05, eps=-0.7)
    x = np.arange(n) * dx
    L = n * dx
    r = np.sqrt((x[:, None, None] - L / 2) ** 2 + (x[None, :, None] - L / 2) ** 2 + (x[None, None, :] + 12.0) ** 2)
    psi = np.cos(r - 12.0 - 0.5 * L)
    orc = O.NeumannOracle(psi, p)
    z, vn, hh, kk = O.neumann_curvature_scan(psi, O.neumann_curvature_fields(orc), dx)
    i = j = n // 2
    rr = r[i, j, z[i, j]]
    assert abs(hh[i, j] * rr / 2 - 1) < 0.02
    assert abs(kk[i, j] * rr * rr - 1) < 0.03


def test_curvature_pass_plane_is_flat():
    """Planar lamellae psi = cos(z - phi): H = K = 0 and v_n = d_t psi / |psi_z|."""
    n = 16
    p = O.Params(n=n, dt=0.05, eps=-0.7)
    z = np.arange(n) * p.dx
    psi = np.broadcast_to(1.3 * np.cos(z - 0.37)[None, None, :], (n, n, n)).copy()
    orc = O.NeumannOracle(psi, p)
    zz, vn, hh, kk = O.neumann_curvature_scan(psi, O.neumann_curvature_fields(orc), p.dx)
    assert (zz >= 0).all() and (zz == zz[0, 0]).all()
    assert np.abs(hh).max() < 1e-12 and np.abs(kk).max() < 1e-12


def test_substrate_zero_sigma_is_plain_neumann():
    """sigma = 0 (the reference's setting) leaves the Neumann step unchanged."""
    n = 16
    psi0 = np.cos(np.arange(n) * 2 * math.pi / 8)[None, None, :] + 0.1 * np.random.default_rng(1).uniform(-1, 1, (n, n, n))
    a = O.NeumannOracle(psi0, O.Params(n=n, dt=0.05, sub_sigma=0.0, sub_z0=2.0))
    b = O.NeumannOracle(psi0, O.Params(n=n, dt=0.05))
    a.run(5)
    b.run(5)
    assert np.array_equal(a.psi, b.psi)


def test_local_amplitude_separable_equals_loops():
    """morphSurfAmp.cpp:1005-1125: the separable window form of the nested
    trapezoids equals the reference's loops."""
    rng = np.random.default_rng(3)
    n = 12
    dx = 2 * math.pi / 8
    psi = np.cos(np.arange(n) * dx)[None, None, :] + 0.3 * rng.uniform(-1, 1, (n, n, n))
    a = O.local_amplitude(psi, dx, 6)
    b = O.local_amplitude_direct(psi, dx, 6)
    assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()


def test_local_amplitude_of_uniform_lamellae_is_one():
    """A box of one wavelength over uniform lamellae holds exactly the reference box's
    weight: psiAvg = 1 everywhere."""
    n = 32
    dx = 2 * math.pi / 8
    psi = np.broadcast_to(1.3 * np.cos(np.arange(n) * dx + 0.4)[None, None, :], (n, n, n))
    m = O.local_amplitude(psi, dx, 8)
    assert np.abs(m[4:-4, 4:-4, 4:-4] - 1).max() < 1e-12


def test_golden_64_regenerates_from_its_seed():
    """The compact 64^3 golden vectors store outputs only: their seeded initial
    conditions must regenerate to the same oracle run."""
    import os
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "neumann_hyperboloid_64.npz"))
    from smectic3d_b200 import ic
    n = 64
    p = O.Params(n=n, dt=float(d["param_dt"]), eps=float(d["param_eps"]))
    o = O.NeumannOracle(ic.hyperboloid(n, p.dx, r0_cells=12.0, seed=12), p)
    o.run(int(d["steps"]))
    assert np.allclose(o.psi[::4, ::4, ::4], d["psi_sub"], rtol=0, atol=1e-13)


def test_sine_transforms_through_the_cosine_pair():
    """RODFT10^3(S) is REDFT10^3 of (-1)^(x+y+z) S read at reversed indices, and
    RODFT01^3(X) is (-1)^(x+y+z) times REDFT01^3 of X reversed: a sine-transform
    Stokes solve on the Neumann box needs no transform beyond the cosine pair."""
    rng = np.random.default_rng(3)
    n = 12
    i = np.arange(n)
    sign = (-1.0) ** (i[:, None, None] + i[None, :, None] + i[None, None, :])
    s = rng.standard_normal((n, n, n))
    a = sfft.dstn(s, type=2)
    b = sfft.dctn(sign * s, type=2)[::-1, ::-1, ::-1]
    assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max()
    x = rng.standard_normal((n, n, n))
    c = sfft.dstn(x, type=3)
    d = sign * sfft.dctn(x[::-1, ::-1, ::-1], type=3)
    assert np.abs(c - d).max() <= 1e-12 * np.abs(c).max()


def test_neumann_oracle_against_the_reference_loop_literally():
    """Two steps of cosFFT/mesabi/cosNoAdvMorph.cpp:216-231,421-442,483-530 with
    REDFT10 / REDFT01 as explicit cosine sums (FFTW's definitions), against the
    vectorised oracle."""
    n, dx, dt, ep, beta, gamma, alpha, q0 = 6, 2 * math.pi / 8, 0.05, -0.3, 2.0, 1.0, 1.0, 1.0
    p = O.Params(n=n, dx=dx, dt=dt, eps=ep, beta=beta, gamma=gamma, alpha=alpha, q0=q0)
    psi0 = np.random.default_rng(9).uniform(-0.6, 0.6, size=(n, n, n))
    kk, nn = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    fwd = 2.0 * np.cos(math.pi * (2 * nn + 1) * kk / (2 * n))                 # REDFT10[k, n]
    inv = np.where(kk == 0, 1.0, 2.0) * np.cos(math.pi * (2 * nn + 1) * kk / (2 * n))
    inv = inv.T                                                                # REDFT01[n, k]

    def t3(m, a):
        return np.einsum("ai,bj,ck,ijk->abc", m, m, m, a)

    vq = [math.pi * i / (dx * n) for i in range(n)]
    c1 = np.empty((n, n, n))
    c2 = np.empty((n, n, n))
    dtd2 = dt / 2
    for i in range(n):
        for j in range(n):
            for k in range(n):
                mq2 = vq[i] ** 2 + vq[j] ** 2 + vq[k] ** 2
                op_sh = alpha * (mq2 - q0 * q0) ** 2
                a_lin = ep - op_sh
                c1[i, j, k] = 1.0 + dtd2 * a_lin
                c2[i, j, k] = 1.0 - dtd2 * a_lin
    scale = 1.0 / (8.0 * n ** 3)
    psi = psi0.copy()
    nq = t3(fwd, beta * psi ** 3 - gamma * psi ** 5)
    for _ in range(2):
        nq_past = nq
        nq = t3(fwd, beta * psi ** 3 - gamma * psi ** 5)
        psiq = t3(fwd, psi)
        psiq = scale * (c1 * psiq + dtd2 * (3.0 * nq - nq_past)) / c2
        psi = t3(inv, psiq)
    orc = O.NeumannOracle(psi0, p)
    orc.run(2)
    assert np.abs(orc.psi - psi).max() <= 1e-13 * np.abs(psi).max()


def test_neumann_velocity_against_the_reference_loop_literally():
    """The Stokes velocity of cosFFT/comet/morphSurfK.cpp (L psi by REDFT01 :686-696,
    wall-one-sided difference gradients :700-766, stress through RODFT10 :760-770,
    the projector with the sine wavenumbers :331-348, 624-631, 862-882, RODFT01)
    with every transform an explicit sum of FFTW's definitions, against the oracle;
    then one advected step built on it, N = beta psi^3 - gamma psi^5 - u . grad psi."""
    n, dx, dt, ep, beta, gamma, alpha, q0, rho, eta = 6, 2 * math.pi / 8, 0.05, -0.3, 2.0, 1.0, 1.0, 1.0, 1.0, 1.0
    p = O.Params(n=n, dx=dx, dt=dt, eps=ep, beta=beta, gamma=gamma, alpha=alpha, q0=q0, rho=rho, eta=eta)
    psi0 = np.random.default_rng(10).uniform(-0.8, 0.8, size=(n, n, n))
    kk, nn = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    cfwd = 2.0 * np.cos(math.pi * (2 * nn + 1) * kk / (2 * n))                      # REDFT10[k, n]
    cinv = (np.where(kk == 0, 1.0, 2.0) * np.cos(math.pi * (2 * nn + 1) * kk / (2 * n))).T  # REDFT01[n, k]
    sfwd = 2.0 * np.sin(math.pi * (2 * nn + 1) * (kk + 1) / (2 * n))                # RODFT10[k, n]
    sinv = (np.where(kk == n - 1, 1.0, 2.0) * np.sin(math.pi * (kk + 1) * (2 * nn + 1) / (2 * n))).T  # RODFT01[n, k]

    def t3(m, a):
        return np.einsum("ai,bj,ck,ijk->abc", m, m, m, a)

    scale = 1.0 / (8.0 * n ** 3)
    vq = np.array([math.pi * i / (dx * n) for i in range(n)])
    vs = np.array([math.pi * (i + 1) / (dx * n) for i in range(n)])
    psi = psi0.copy()
    psiq = t3(cfwd, psi)
    op_sh = np.empty((n, n, n))
    cm1 = np.empty((n, n, n))
    cm2 = np.empty((3, n, n, n))
    for i in range(n):
        for j in range(n):
            for k in range(n):
                op_sh[i, j, k] = scale * alpha * (vq[i] ** 2 + vq[j] ** 2 + vq[k] ** 2 - q0 * q0) ** 2
                mq2 = vs[i] ** 2 + vs[j] ** 2 + vs[k] ** 2
                cm1[i, j, k] = scale / (rho * eta * mq2)
                cm2[:, i, j, k] = (vs[i] / mq2, vs[j] / mq2, vs[k] / mq2)
    psi_sh = t3(cinv, op_sh * psiq)
    grad = np.empty((3, n, n, n))
    for ax in range(3):
        a = np.moveaxis(psi, ax, 0)
        g = np.empty_like(a)
        for i in range(n):
            if 0 < i < n - 1:
                g[i] = (a[i + 1] - a[i - 1]) / (2 * dx)
            elif i == 0:
                g[i] = 2 * (a[1] - a[0]) / (2 * dx)
            else:
                g[i] = 2 * (a[i] - a[i - 1]) / (2 * dx)
        grad[ax] = np.moveaxis(g, 0, ax)
    sq = np.array([t3(sfwd, psi_sh * grad[c]) for c in range(3)])
    dot = vs[:, None, None] * sq[0] + vs[None, :, None] * sq[1] + vs[None, None, :] * sq[2]
    u = np.array([t3(sinv, cm1 * (sq[c] - cm2[c] * dot)) for c in range(3)])
    orc = O.NeumannOracle(psi0, p, advect=True)
    uo, go, lo = orc.velocity(O.dct3d(psi0))
    assert np.abs(np.array(go) - grad).max() <= 1e-13 * np.abs(grad).max()
    assert np.abs(np.array(uo) - u).max() <= 1e-12 * np.abs(u).max()
    assert np.abs(u).max() > 1e-6
    # one advected step: the history N-hat has no advection, the current one has
    nr = beta * psi ** 3 - gamma * psi ** 5
    nq_past = t3(cfwd, nr)
    nq = t3(cfwd, nr - (u * grad).sum(axis=0))
    c1 = 1.0 + dt / 2 * (ep - op_sh / scale)
    c2 = 1.0 - dt / 2 * (ep - op_sh / scale)
    psi1 = t3(cinv, scale * (c1 * psiq + dt / 2 * (3.0 * nq - nq_past)) / c2)
    orc.step()
    assert np.abs(orc.psi - psi1).max() <= 1e-12 * np.abs(psi1).max()


def test_periodic_oracle_against_the_reference_loop_literally():
    """Two plain steps of periodicFFT/pf3dVal.cpp:129-299 (k-vectors pf3d.cpp:162-190,
    tables :195-222, update :471-481) with the 3-D transform written as explicit
    complex exponential sums over the full spectrum, against the vectorised
    oracle (its r2c / c2r half-spectrum form)."""
    n, dx, dt, ep, beta, gamma, alpha, q0 = 6, 2 * math.pi / 8, 0.05, -0.3, 2.0, 1.0, 1.0, 1.0
    p = O.Params(n=n, dx=dx, dt=dt, eps=ep, beta=beta, gamma=gamma, alpha=alpha, q0=q0)
    psi0 = np.random.default_rng(10).uniform(-0.6, 0.6, size=(n, n, n))
    kk, nn = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    fwd = np.exp(-2j * math.pi * kk * nn / n)          # FFTW forward, unnormalised
    bwd = np.exp(+2j * math.pi * kk * nn / n).T        # FFTW backward, unnormalised

    def t3(m, a):
        return np.einsum("ai,bj,ck,ijk->abc", m, m, m, a)

    vq = [2 * math.pi * i / (dx * n) if i <= n // 2 else -(n - i) * 2 * math.pi / (dx * n) for i in range(n)]
    c1 = np.empty((n, n, n))
    c2 = np.empty((n, n, n))
    dtd2 = dt / 2
    for i in range(n):
        for j in range(n):
            for k in range(n):
                mq2 = vq[i] ** 2 + vq[j] ** 2 + vq[k] ** 2
                a_lin = ep - alpha * (mq2 - q0 * q0) ** 2
                c1[i, j, k] = 1.0 + dtd2 * a_lin
                c2[i, j, k] = 1.0 - dtd2 * a_lin
    scale = 1.0 / n ** 3
    psi = psi0.copy()
    nq_past = t3(fwd, beta * psi ** 3 - gamma * psi ** 5)
    for _ in range(2):
        nq = t3(fwd, beta * psi ** 3 - gamma * psi ** 5)
        psiq = t3(fwd, psi)
        psiq = scale * (c1 * psiq + dtd2 * (3.0 * nq - nq_past)) / c2
        psi = t3(bwd, psiq).real
        nq_past = nq
    orc = O.PeriodicOracle(psi0, p)
    orc.run(2)
    assert np.abs(orc.psi - psi).max() <= 1e-13 * np.abs(psi).max()
