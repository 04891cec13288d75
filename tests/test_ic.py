"""Initial-condition generators against literal scalar loops written the way
the reference writes them (periodicFFT/pf3d.cpp:302-324,
cosFFT/mesabi/cosNoAdvMorph.cpp:289-331, periodicFFT/pf3dMorph.cpp:331-376,
periodicFFT/pf3dVal.cpp:219-229), and the seeded synthetic ICs of the
benchmark workloads against their formulas."""
import math

import numpy as np

import smectic3d_b200 as S

N = 16
DX = 2 * math.pi / 8


def test_pf3d_lamellae_matches_the_loop():
    amp, qi, q0, kmin, kmax = 1.2441, 0.5, 1.0, 2, 14
    ref = np.zeros((N, N, N))
    for i in range(N):
        for j in range(N):
            for k in range(N):
                if k > kmin and k < kmax:
                    ref[i, j, k] = (amp * math.cos(q0 * k * DX)
                                    + amp * 0.1 * math.sin(q0 * k * DX) * (math.cos(qi * i * DX) + math.cos(qi * j * DX)))
    got = S.ic.pf3d_lamellae(N, DX, kmin=kmin, kmax=kmax)
    assert np.abs(got - ref).max() <= 1e-14
    # the reference's own bounds at its own size
    full = S.ic.pf3d_lamellae(256, DX)
    assert not full[:, :, 24].any() and full[:, :, 25].any() and full[:, :, 231].any() and not full[:, :, 232].any()


def _morph_loop(mid, a_e, b_e, amp, zfun, keep):
    ref = np.zeros((N, N, N))
    for i in range(N):
        for j in range(N):
            for k in range(N):
                if not keep(k):
                    continue
                xs, ys, zs = i - mid, j - mid, zfun(k)
                ds = math.sqrt(xs * xs + ys * ys)
                if ds < mid:
                    if math.sqrt(((ds - mid) / a_e) ** 2 + (zs / b_e) ** 2) > 1:
                        ref[i, j, k] = 0.0
                    else:
                        ref[i, j, k] = amp * math.cos(DX * math.sqrt(((b_e / a_e) * (ds - mid)) ** 2 + zs * zs))
                else:
                    ref[i, j, k] = amp * math.cos(zs * DX) if abs(zs) < b_e else 0.0
    return ref


def test_cos_bottom_hyperboloid_matches_the_loop():
    a_e, b_e, mid = 9.75, 11.75, N / 2
    ref = _morph_loop(mid, a_e, b_e, 1.328, lambda k: k, lambda k: k < b_e + 1)
    got = S.ic.cos_bottom_hyperboloid(N, DX, a_e=a_e, b_e=b_e)
    assert np.abs(got - ref).max() <= 1e-14


def test_pf3dmorph_torus_matches_the_loop():
    a_e, b_e, mid = 245.0 * N / 512, 180.0 * N / 512, N / 2
    kmin, kmax = 62 * N / 512, 450 * N / 512
    ref = _morph_loop(mid, a_e, b_e, 1.328, lambda k: k - mid, lambda k: kmin < k < kmax)
    got = S.ic.pf3dmorph_torus(N, DX)
    assert np.abs(got - ref).max() <= 1e-14


def test_pf3dval_mode():
    got = S.ic.pf3dval_mode(N, DX, mqz=2.0)
    k = np.arange(N)
    assert np.abs(got - 1e-4 * np.cos(2.0 * k * DX)[None, None, :]).max() <= 1e-19


def test_workload_hyperboloid_formula_and_seed():
    r0 = 20 * DX
    got = S.ic.hyperboloid(N, DX, noise_amp=0.0)
    for (i, j, k) in [(0, 0, 0), (3, 5, 7), (8, 8, 8), (15, 2, 11)]:
        x, y, z = (i - N / 2) * DX, (j - N / 2) * DX, (k - N / 2) * DX
        s = math.sqrt(max(x * x + y * y - z * z + r0 * r0, 0.0))
        assert abs(got[i, j, k] - 0.5 * math.cos(s)) <= 1e-15
    a, b = S.ic.hyperboloid(N, DX, seed=4), S.ic.hyperboloid(N, DX, seed=4)
    assert np.array_equal(a, b)
    assert 0 < np.abs(a - got).max() <= 1e-3


def test_noise_and_batches():
    a = S.ic.noise(N, 7, amp=0.1)
    assert a.shape == (N, N, N) and np.abs(a).max() <= 0.1 and np.array_equal(a, S.ic.noise(N, 7, amp=0.1))
    b = S.ic.noise_batch(N, [7, 8])
    assert b.shape == (2, N, N, N) and np.array_equal(b[0], a) and not np.array_equal(b[0], b[1])


def test_undulated_lamellae_formula():
    got = S.ic.undulated_lamellae(N, DX, amp=1.3, seed=2)
    phi = np.random.default_rng(2).uniform(0.0, 2.0 * math.pi)
    for (i, j, k) in [(0, 0, 0), (5, 9, 3), (15, 15, 15)]:
        h = 2 * DX * math.sin(2 * math.pi * i * DX / (64 * DX) + phi)
        assert abs(got[i, j, k] - 1.3 * math.cos(k * DX - h)) <= 1e-14
