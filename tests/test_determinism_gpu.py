"""Bitwise reproducibility: two handles advanced side by side from the same state
hold bitwise identical fields after every checked step.

Every reduction of the library has a fixed order and no kernel uses atomics on
field data, so any difference between two runs is a race.  The advected Neumann
step at 256^3 runs three row-first plane passes (stress components, clusters of
8) per step; a missing barrier between the twiddle staging and their first
row transform once made about one step in fifty differ.  The checks run at the
sizes where the passes are clustered (256^3) and with enough steps for a rare
race to show.
"""
import numpy as np
import pytest

import smectic3d_b200 as S

pytestmark = pytest.mark.gpu


def _lockstep(params, psi0, steps, every):
    with S.Solver(params) as a, S.Solver(params) as b:
        a.set_psi(psi0)
        b.set_psi(psi0)
        for k in range(1, steps + 1):
            a.step(1)
            b.step(1)
            if k % every == 0 or k == steps:
                pa, pb = a.get_psi(), b.get_psi()
                nd = int(np.count_nonzero(pa != pb))
                assert nd == 0, f"step {k}: {nd} points differ, max {float(np.max(np.abs(pa - pb)))}"


def test_advected_neumann_256_fp32_is_bitwise_reproducible():
    p = S.Params(n=256, boundary="neumann", precision="fp32", dt=0.05, eps=-0.75, advection=True)
    _lockstep(p, S.ic.noise(256, 0), steps=120, every=10)


def test_advected_periodic_256_fp32_is_bitwise_reproducible():
    p = S.Params(n=256, boundary="periodic", precision="fp32", dt=0.05, eps=-0.75, advection=True)
    _lockstep(p, S.ic.noise(256, 1), steps=60, every=20)


@pytest.mark.parametrize("boundary", ["neumann", "periodic"])
def test_plain_256_fp32_graph_runs_are_bitwise_reproducible(boundary):
    p = S.Params(n=256, boundary=boundary, precision="fp32", dt=0.05, eps=-0.75)
    psi0 = S.ic.noise(256, 2)
    outs = []
    for _ in range(3):
        with S.Solver(p) as s:
            s.set_psi(psi0)
            s.step(400)  # CUDA-graph replay of 16-step chunks
            outs.append(s.get_psi())
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])


def test_adjoint_is_bitwise_reproducible():
    """The reverse sweep ends with an inverse-only pencil pass (lambda^0 to real
    space) whose first transform reads the staged twiddles right away."""
    n = 128
    p = S.Params(n=n, boundary="periodic", precision="fp32", dt=0.05, eps=-0.75)
    psi0 = S.ic.noise(n, 3)
    lam = np.zeros_like(psi0)
    lam[n // 2, :, :] = 1.0
    res = []
    for _ in range(3):
        with S.Solver(p) as s:
            res.append(s.adjoint(psi0, 40, lam, ckpt_every=10))
    for r in res[1:]:
        for x, y in zip(r, res[0]):
            assert np.array_equal(x, y)


def test_batched_replicas_graph_runs_are_bitwise_reproducible():
    b = 16
    p = S.Params(n=64, batch=b, boundary="periodic", precision="fp32", dt=0.05, eps=-0.75,
                 eps_per_replica=tuple(np.linspace(-0.9, -0.5, b)))
    psi0 = S.ic.noise_batch(64, range(b))
    outs = []
    for _ in range(2):
        with S.Solver(p) as s:
            s.set_psi(psi0)
            s.step(320)
            outs.append(s.get_psi())
    assert np.array_equal(outs[0], outs[1])


def test_advected_neumann_256_fp64_is_bitwise_reproducible():
    """FP64 cosine plane passes at 256^3 read their twiddles through L1 (no staging)."""
    p = S.Params(n=256, boundary="neumann", precision="fp64", dt=0.05, eps=-0.75, advection=True)
    _lockstep(p, S.ic.noise(256, 4), steps=20, every=10)


def test_surface_step_is_bitwise_reproducible():
    p = S.Params(n=256, boundary="periodic", precision="fp32", dt=0.05, eps=-0.75, advection=True)
    psi0 = S.ic.noise(256, 5)
    outs = []
    for _ in range(2):
        with S.Solver(p) as s:
            s.set_psi(psi0)
            s.step(3)
            outs.append(s.surface_step())
    for x, y in zip(outs[0], outs[1]):
        assert np.array_equal(x, y, equal_nan=True) if x.dtype.kind == "f" else np.array_equal(x, y)


@pytest.mark.parametrize("boundary", ["neumann", "periodic"])
def test_l1_monitor_graph_replay_matches_direct_steps(boundary):
    """With the L1 monitor on, step(n) replays the step graph between the
    monitored steps; single steps take every step directly.  Both give the same
    state and the same L1 values bit for bit."""
    n = 128
    p = S.Params(n=n, boundary=boundary, precision="fp32", dt=0.05, eps=-0.75, l1_interval=20)
    psi0 = S.ic.noise(n, 6, amp=0.3)
    with S.Solver(p) as a, S.Solver(p) as b:
        a.set_psi(psi0)
        b.set_psi(psi0)
        la, lb = [], []
        for _ in range(3):
            a.step(47)
            la.append(a.l1())
            for _ in range(47):
                b.step(1)
            lb.append(b.l1())
        assert np.array_equal(a.get_psi(), b.get_psi())
        for x, y in zip(la, lb):
            assert np.array_equal(np.asarray(x[0]), np.asarray(y[0])) and x[1] == y[1]
