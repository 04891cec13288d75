"""torch.autograd over the time loop (smectic3d_b200.torch_adjoint): its gradients
are the discrete adjoint's, and they match central finite differences."""
import dataclasses

import numpy as np
import pytest

import smectic3d_b200 as S

pytestmark = pytest.mark.gpu


def test_autograd_matches_sh_adjoint_and_finite_differences():
    torch = pytest.importorskip("torch")
    from smectic3d_b200.torch_adjoint import sh_evolve
    n, steps, k = 16, 10, 4
    p = S.Params(n=n, precision="fp64", dt=0.05)
    z = np.arange(n) * p.dx
    init = 1.3 * np.cos(z)[None, None, :] + S.ic.noise(n, 3, 0.1)
    target = torch.tensor(np.broadcast_to(0.5 * np.cos(1.05 * z)[None, None, :], (n, n, n)).copy())
    psi0 = torch.tensor(init, requires_grad=True)
    eps = torch.tensor(-0.7, dtype=torch.float64, requires_grad=True)
    q0 = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    loss = 0.5 * ((sh_evolve(psi0, eps, q0, p, steps, ckpt_every=k) - target) ** 2).sum()
    loss.backward()

    pe = dataclasses.replace(p, eps=-0.7, q0=1.0)
    with S.Solver(pe) as s:
        s.set_psi(init)
        s.step(steps)
        lam = s.get_psi() - target.numpy()
        ge, gq, gp = s.adjoint(init, steps, lam, ckpt_every=k)
    assert abs(eps.grad.item() - ge[0]) <= 1e-12 * abs(ge[0])
    assert abs(q0.grad.item() - gq[0]) <= 1e-12 * abs(gq[0])
    assert np.allclose(psi0.grad.numpy(), gp, rtol=0, atol=1e-12 * np.abs(gp).max())

    def loss_at(e):
        with S.Solver(dataclasses.replace(p, eps=e, q0=1.0)) as s:
            s.set_psi(init)
            s.step(steps)
            return 0.5 * float(((s.get_psi() - target.numpy()) ** 2).sum())
    h = 1e-4
    fd = (loss_at(-0.7 + h) - loss_at(-0.7 - h)) / (2 * h)
    assert abs(eps.grad.item() - fd) <= 1e-4 * abs(fd)


def test_autograd_on_device_tensors():
    """Inputs on cuda:0 get their gradients on cuda:0, equal to the host case."""
    torch = pytest.importorskip("torch")
    from smectic3d_b200.torch_adjoint import sh_evolve
    n, steps = 16, 4
    p = S.Params(n=n, precision="fp64", dt=0.05)
    init = torch.tensor(S.ic.noise(n, 5, 0.2))
    grads = []
    for dev in ("cpu", "cuda:0"):
        psi0 = init.clone().to(dev).requires_grad_(True)
        eps = torch.tensor(-0.3, dtype=torch.float64, device=dev, requires_grad=True)
        q0 = torch.tensor(1.0, dtype=torch.float64, device=dev, requires_grad=True)
        out = sh_evolve(psi0, eps, q0, p, steps, ckpt_every=2)
        assert out.device == psi0.device
        (out ** 2).sum().backward()
        assert psi0.grad.device == psi0.device and eps.grad.device == eps.device and q0.grad.device == q0.device
        grads.append((psi0.grad.cpu().numpy(), eps.grad.item(), q0.grad.item()))
    assert np.array_equal(grads[0][0], grads[1][0])
    assert grads[0][1] == grads[1][1] and grads[0][2] == grads[1][2]
