"""The adjoint on its own configuration (C5): periodic 128^3, FP32 forward with
FP64 gradient sums, eps = -0.75, dt = 0.05, T = 1000 steps, a checkpoint every
50, loss L = 1/2 ||psi_T - target||^2 with target 0.5 cos(1.05 z).

Gradients with respect to eps and q0 are checked against central finite
differences (h = 1e-4) of the FP64 forward run on the GPU and against the FP64
adjoint; the psi0 gradient by a directional difference along a seeded
direction.  All to 1e-4 relative.  The finite differences are formed from the
two final states, L(+) - L(-) = <psi_T(+) - psi_T(-), (psi_T(+) + psi_T(-))/2 - target>,
so that the constant 1/2 ||target||^2 does not swamp a loss that changes by
far less than FP64's resolution of it (the noise IC decays to about
1e-18 over T).  C5' starts from reference-amplitude lamellae
1.328 cos(z) + that noise instead.
"""
import dataclasses

import numpy as np
import pytest

import smectic3d_b200 as S
from smectic3d_b200 import _lib as L

pytestmark = pytest.mark.gpu

N, T, K, H = 128, 1000, 50, 1e-4


def setup(case, prec="fp32"):
    p = S.Params(n=N, precision=prec, dt=0.05, eps=-0.75)
    z = np.arange(N) * p.dx
    psi0 = S.ic.noise(N, 0)
    if case == "c5p_lamellae":
        psi0 = psi0 + 1.328 * np.cos(z)[None, None, :]
    target = np.broadcast_to(0.5 * np.cos(1.05 * z)[None, None, :], (N, N, N)).copy()
    return p, psi0, target


def final_state(p, psi0):
    with S.Solver(p) as s:
        s.set_psi(psi0)
        s.step(T)
        return s.get_psi()


def fd(p, psi0, target, field, h=H, direction=None):
    """Central difference of L along eps, q0 or a direction of psi0 (FP64 forward)."""
    q = dataclasses.replace(p, precision="fp64")
    if field == "psi0":
        plus, minus = final_state(q, psi0 + h * direction), final_state(q, psi0 - h * direction)
    else:
        v = getattr(q, field)
        plus = final_state(dataclasses.replace(q, **{field: v + h}), psi0)
        minus = final_state(dataclasses.replace(q, **{field: v - h}), psi0)
    d = plus - minus
    return float(np.vdot(d, 0.5 * (plus + minus) - target)) / (2 * h)


def gradients(p, psi0, target):
    with S.Solver(p) as s:
        s.adjoint_forward(psi0, T, K)
        psi_t = s.get_psi()
        ge, gq, gp = s.adjoint_backward(psi_t - target)
        # the handle still holds psi^T: a second backward over the same checkpoints agrees
        ge2, gq2, _ = s.adjoint_backward(psi_t - target)
        assert ge2[0] == ge[0] and gq2[0] == gq[0]
        assert np.array_equal(s.get_psi(), psi_t)
    return ge[0], gq[0], gp


def close(a, b, tol=1e-4):
    return abs(a - b) <= tol * abs(b)


# The noise IC decays by e^-37 over T: its gradients need the FP32 fields' update
# in FP64 (fp32_u64), whose multipliers carry no per-step bias, to stay within
# 1e-4 of the differences; the lamellae run in either FP32 form.
@pytest.mark.parametrize("case,prec", [("c5_noise", "fp32_u64"), ("c5p_lamellae", "fp32"),
                                       ("c5p_lamellae", "fp32_u64")])
def test_c5_gradients_against_fd_and_fp64_adjoint(case, prec):
    p, psi0, target = setup(case, prec)
    ge32, gq32, gp32 = gradients(p, psi0, target)
    ge64, gq64, gp64 = gradients(dataclasses.replace(p, precision="fp64"), psi0, target)
    fe, fq = fd(p, psi0, target, "eps"), fd(p, psi0, target, "q0")
    direction = np.random.default_rng(5).uniform(-1.0, 1.0, size=psi0.shape)
    fp = fd(p, psi0, target, "psi0", direction=direction)
    dp32, dp64 = float(np.vdot(gp32, direction)), float(np.vdot(gp64, direction))
    report = dict(ge32=ge32, ge64=ge64, fd_eps=fe, gq32=gq32, gq64=gq64, fd_q0=fq, dpsi32=dp32, dpsi64=dp64,
                  fd_psi0=fp, gpsi_rel=float(np.linalg.norm(gp32 - gp64) / np.linalg.norm(gp64)))
    print(case, prec, report)
    # FP64 adjoint against the differences
    assert close(ge64, fe) and close(gq64, fq) and close(dp64, fp), report
    # FP32 forward, FP64 sums: against the differences and the FP64 adjoint
    assert close(ge32, fe) and close(gq32, fq) and close(dp32, fp), report
    assert close(ge32, ge64) and close(gq32, gq64) and close(dp32, dp64), report
    assert np.linalg.norm(gp32 - gp64) <= 1e-4 * np.linalg.norm(gp64), report


def test_backward_without_forward_is_refused():
    p = S.Params(n=16, precision="fp32", dt=0.05, eps=-0.75)
    psi0 = S.ic.noise(16, 1)
    with S.Solver(p) as s:
        s.set_psi(psi0)
        with pytest.raises(S.ShError) as e:
            s.adjoint_backward(psi0)
        assert e.value.code == L.SH_ESTATE
        s.adjoint_forward(psi0, 4, 2)
        s.step(1)  # the state moved on: the checkpoints no longer end here
        with pytest.raises(S.ShError):
            s.adjoint_backward(psi0)
