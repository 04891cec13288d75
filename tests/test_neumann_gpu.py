"""GPU parity of the Neumann-only parts of the path against the FP64 oracle:
the substrate penalty (cosFFT/comet/cosNoAdvMorph.cpp:67-74, 591-623), the
curvature pass (cosFFT/comet/cosNoAdvMorphCurv.cpp:742-965) and the advected
step with the sine-transform Stokes velocity (cosFFT/comet/morphSurfK.cpp)."""
import math

import numpy as np
import pytest

import smectic3d_b200 as S
from oracle import sh_oracle as O
from smectic3d_b200 import _lib as L

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "fp32": 1e-5}


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def oracle_params(p: S.Params) -> O.Params:
    return O.Params(n=p.n, dx=p.dx, dt=p.dt, eps=p.eps, beta=p.beta, gamma=p.gamma, alpha=p.alpha, q0=p.q0,
                    eta=p.eta, rho=p.rho, nonlinearity=p.nonlinearity, scheme=p.scheme, w_mid=p.w_mid,
                    sub_sigma=p.sub_sigma, sub_z0=p.sub_z0)


def undulated(n, dx, amp=0.9, phase=0.37):
    """Lamellae along z displaced by a Neumann-compatible height field, with
    off-grid phases so that no grid value of psi is exactly 0 or 0.7."""
    c = np.arange(n) * dx
    L = n * dx
    h = amp * (np.cos(2 * np.pi * c / L + 0.3)[:, None, None] * np.cos(np.pi * c / L + 0.2)[None, :, None])
    return 1.3 * np.cos(c[None, None, :] - h - phase)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("z0", [1e-4, 2.0])
@pytest.mark.parametrize("n", [32, 64])
def test_substrate_matches_oracle(n, z0, prec):
    """wall(z) = sigma exp(-z/z0) times the in-plane Laplacian of psi^n joins N;
    z0 = 1e-4 (the reference's value) leaves only the bottom plane, 2.0 a
    band of planes."""
    p = S.Params(n=n, boundary="neumann", precision=prec, dt=0.05, eps=-0.7, sub_sigma=0.5, sub_z0=z0)
    psi0 = S.ic.cos_bottom_hyperboloid(n, p.dx) + S.ic.noise(n, 3, 0.05)
    orc = O.NeumannOracle(psi0, oracle_params(p))
    orc.run(40)
    with S.Solver(p) as s:
        s.set_psi(psi0)
        s.step(40)
        psi = s.get_psi()
    assert rel(psi, orc.psi) <= TOL[prec]
    # and the term matters: without it the state differs far beyond the tolerance
    q = O.NeumannOracle(psi0, oracle_params(S.Params(n=n, boundary="neumann", dt=0.05, eps=-0.7)))
    q.run(40)
    assert rel(q.psi, orc.psi) > 1e3 * TOL["fp64"]


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("n", [32, 64])
def test_curvature_pass_matches_oracle(n, prec):
    p = S.Params(n=n, boundary="neumann", precision=prec, dt=0.05, eps=-0.7)
    psi0 = undulated(n, p.dx)
    orc = O.NeumannOracle(psi0, oracle_params(p))
    orc.run(3)
    f = O.neumann_curvature_fields(orc)
    zo, vo, ho, ko = O.neumann_curvature_scan(orc.psi, f, p.dx)
    orc.step()
    with S.Solver(p) as s:
        s.set_psi(psi0)
        s.step(3)
        z, vn, hh, kk = s.surface_step()
        assert rel(s.get_psi(), orc.psi) <= TOL[prec]  # the pass also took the step
    found = zo >= 0
    assert found.mean() > 0.9
    same = z == zo
    assert same.mean() >= (1.0 if prec == "fp64" else 0.99)
    m = same & found
    tol = 1e-8 if prec == "fp64" else 2e-3
    for got, ref in ((vn, vo), (hh, ho), (kk, ko)):
        scale = max(np.abs(ref[m]).max(), 1e-3)
        assert np.abs(got[m] - ref[m]).max() <= tol * scale
    assert np.abs(ko[m]).max() > 1e-4  # doubly curved
    assert np.isnan(hh[z < 0]).all()


def test_curvature_pass_sphere():
    """Known answer: spherical level sets psi = cos(r - R) centred below the box:
    H = 2/r and K = 1/r^2 at the crossing, to the accuracy of the reference's
    difference gradients (dx = 2 pi / 32)."""
    n = 64
    dx = 2 * math.pi / 32
    p = S.Params(n=n, dx=dx, boundary="neumann", precision="fp64", dt=0.01, eps=-0.7)
    x = np.arange(n) * dx
    L = n * dx
    r = np.sqrt((x[:, None, None] - L / 2) ** 2 + (x[None, :, None] - L / 2) ** 2 + (x[None, None, :] + 12.0) ** 2)
    psi0 = np.cos(r - 12.0 - 0.5 * L - 0.11)
    with S.Solver(p) as s:
        s.set_psi(psi0)
        z, vn, hh, kk = s.surface_step()
    for i, j in ((n // 2, n // 2), (n // 2 + 5, n // 2 - 7)):
        assert z[i, j] >= 0
        rr = r[i, j, z[i, j]]
        assert abs(hh[i, j] * rr / 2 - 1) < 0.02
        assert abs(kk[i, j] * rr * rr - 1) < 0.03


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("n", [32, 64])
def test_spectral_curvature_pass_matches_oracle(n, prec):
    """curvature = "spectral": the gradient and mixed derivatives are the exact
    derivatives of the cosine series (sine series through the signed cosine pair
    on the GPU), against the oracle's scipy DST-III evaluation."""
    p = S.Params(n=n, boundary="neumann", precision=prec, dt=0.05, eps=-0.7, curvature="spectral")
    psi0 = undulated(n, p.dx)
    orc = O.NeumannOracle(psi0, oracle_params(p))
    orc.run(3)
    f = O.neumann_curvature_fields(orc)
    sp = O.neumann_spectral_derivatives(orc.psi, p.dx)
    zo, vo, ho, ko = O.neumann_curvature_scan(orc.psi, f, p.dx, spectral=sp)
    with S.Solver(p) as s:
        s.set_psi(psi0)
        s.step(3)
        z, vn, hh, kk = s.surface_step()
    found = zo >= 0
    assert found.mean() > 0.9
    same = z == zo
    assert same.mean() >= (1.0 if prec == "fp64" else 0.99)
    m = same & found
    tol = 1e-8 if prec == "fp64" else 2e-3
    for got, ref in ((vn, vo), (hh, ho), (kk, ko)):
        scale = max(np.abs(ref[m]).max(), 1e-3)
        assert np.abs(got[m] - ref[m]).max() <= tol * scale


def test_curvature_pass_sphere_spectral_beats_differences():
    """The sphere known answer (H = 2/r, K = 1/r^2) with both gradient forms: the
    spectral one is closer at every probed column."""
    n = 64
    dx = 2 * math.pi / 32
    x = np.arange(n) * dx
    L = n * dx
    r = np.sqrt((x[:, None, None] - L / 2) ** 2 + (x[None, :, None] - L / 2) ** 2 + (x[None, None, :] + 12.0) ** 2)
    psi0 = np.cos(r - 12.0 - 0.5 * L - 0.11)
    err = {}
    for form in ("difference", "spectral"):
        p = S.Params(n=n, dx=dx, boundary="neumann", precision="fp64", dt=0.01, eps=-0.7, curvature=form)
        with S.Solver(p) as s:
            s.set_psi(psi0)
            z, vn, hh, kk = s.surface_step()
        e = []
        for i, j in ((n // 2, n // 2), (n // 2 + 5, n // 2 - 7), (n // 2 - 10, n // 2 + 3)):
            assert z[i, j] >= 0
            rr = r[i, j, z[i, j]]
            e.append((abs(hh[i, j] * rr / 2 - 1), abs(kk[i, j] * rr * rr - 1)))
        err[form] = np.array(e)
    assert (err["spectral"] < err["difference"]).all(), err
    assert err["spectral"].max() < 5e-3, err


@pytest.mark.parametrize("boundary,prec", [("neumann", "fp64"), ("neumann", "fp32"), ("periodic", "fp64")])
def test_local_amplitude_matches_oracle(boundary, prec):
    """sh_local_amplitude (morphSurfAmp.cpp:1005-1125) on the handle's own psi
    against the oracle's separable trapezoids; the map is FP64 either way."""
    n = 64
    p = S.Params(n=n, boundary=boundary, precision=prec, dt=0.05, eps=-0.7)
    with S.Solver(p) as s:
        s.set_psi(undulated(n, p.dx) + S.ic.noise(n, 4, 0.1))
        s.step(5)
        psi = s.get_psi()
        # Nw = grid cells per wavelength (dx = 2 pi / 8): the box spans one wavelength
        amp = s.local_amplitude(8)
        with pytest.raises(S.ShError):
            s.local_amplitude(44)  # 3 (nw/2) > n - 1
    ref = O.local_amplitude(psi, p.dx, 8)
    assert np.abs(amp - ref).max() <= 1e-12 * np.abs(ref).max()
    assert 0.5 < np.median(amp) < 1.5


def test_substrate_checkpoint_roundtrip_is_bit_exact():
    """The substrate term is recomputed from the state each step: a restored
    checkpoint continues bit for bit."""
    n = 32
    p = S.Params(n=n, boundary="neumann", precision="fp64", dt=0.05, eps=-0.7, sub_sigma=0.5, sub_z0=2.0)
    with S.Solver(p) as s:
        s.set_psi(S.ic.cos_bottom_hyperboloid(n, p.dx) + S.ic.noise(n, 5, 0.05))
        s.step(3)
        blob = s.checkpoint()
        s.step(5)
        a = s.get_psi()
        s.restore(blob)
        s.step(5)
        b = s.get_psi()
    assert np.array_equal(a, b)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_batched_curvature_and_amplitude_match_single_replicas(prec):
    """Replicas are independent through the curvature pass and the amplitude map:
    a batch of two gives what two single-replica handles give."""
    n = 32
    p1 = S.Params(n=n, boundary="neumann", precision=prec, dt=0.05, eps=-0.7)
    ics = [undulated(n, p1.dx), undulated(n, p1.dx, amp=0.6, phase=0.21)]
    single = []
    for ic in ics:
        with S.Solver(p1) as s:
            s.set_psi(ic)
            s.step(2)
            amp = s.local_amplitude(8)
            z, vn, hh, kk = s.surface_step()
            single.append((amp, z, vn, hh, kk, s.get_psi()))
    p2 = S.Params(n=n, batch=2, boundary="neumann", precision=prec, dt=0.05, eps=-0.7)
    with S.Solver(p2) as s:
        s.set_psi(np.stack(ics))
        s.step(2)
        amp = s.local_amplitude(8)
        z, vn, hh, kk = s.surface_step()
        psi = s.get_psi()
    for r in range(2):
        a1, z1, v1, h1, k1, p1r = single[r]
        assert np.array_equal(z[r], z1)
        m = z1 >= 0
        for got, ref in ((amp[r], a1), (vn[r][m], v1[m]), (hh[r][m], h1[m]), (kk[r][m], k1[m]), (psi[r], p1r)):
            assert np.allclose(got, ref, rtol=1e-12 if prec == "fp64" else 1e-5, atol=1e-12)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("n", [16, 32, 64, 128])
def test_advected_neumann_matches_oracle(n, prec):
    """Neumann step with the Stokes velocity of morphSurfK.cpp (RODFT10/01 through
    the signed cosine pair on the GPU): psi after 12 steps and the velocity of
    the final state against the oracle."""
    p = S.Params(n=n, boundary="neumann", advection=True, precision=prec, dt=0.02, eps=-0.7, eta=0.5)
    psi0 = undulated(n, p.dx) + S.ic.noise(n, 21, 0.05)
    orc = O.NeumannOracle(psi0, oracle_params(p), advect=True)
    orc.run(12)
    uo, _, _ = orc.velocity(O.dct3d(orc.psi))
    with S.Solver(p) as s:
        s.set_psi(psi0)
        s.step(12)
        assert rel(s.get_psi(), orc.psi) <= TOL[prec]
        u = s.velocity()
    for c in range(3):
        assert rel(u[c], uo[c]) <= (1e-10 if prec == "fp64" else 1e-4), c
    assert max(np.abs(x).max() for x in uo) > 1e-4  # the flow is not trivially zero


def test_advected_neumann_256_few_steps():
    """The Neumann advected step at 256^3 (FP32) against the oracle for two steps."""
    n = 256
    p = S.Params(n=n, boundary="neumann", advection=True, precision="fp32", dt=0.02, eps=-0.75)
    psi0 = S.ic.hyperboloid(n, p.dx, amp=1.328, seed=0)
    orc = O.NeumannOracle(psi0, oracle_params(p), advect=True)
    orc.run(2)
    with S.Solver(p) as s:
        s.set_psi(psi0)
        s.step(2)
        assert rel(s.get_psi(), orc.psi) <= TOL["fp32"]


def test_advected_neumann_refuses_curvature_pass():
    p = S.Params(n=16, boundary="neumann", advection=True, precision="fp64")
    with S.Solver(p) as s:
        s.set_psi(undulated(16, p.dx))
        with pytest.raises(S.ShError) as e:
            s.surface_step()
        assert e.value.code == L.SH_EUNSUPPORTED
