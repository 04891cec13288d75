"""Every built cluster size of the plane pass computes the same step: the
transforms do the same arithmetic whatever CTA owns a line, so the variants of
one shape agree to FP32 rounding (the exchange layouts differ between them)."""
import numpy as np
import pytest

import smectic3d_b200 as S

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("boundary", ["neumann", "periodic"])
@pytest.mark.parametrize("n,variants", [(64, (1, 2)), (128, (1, 2, 4)), (256, (4, 8, 16))])
def test_cluster_sizes_agree(n, variants, boundary):
    p = S.Params(n=n, boundary=boundary, precision="fp32")
    psi0 = S.ic.undulated_lamellae(n, p.dx, amp=1.3, seed=0)
    outs = {}
    for v in variants:
        with S.Solver(S.Params(n=n, boundary=boundary, precision="fp32", variant=v)) as s:
            s.set_psi(psi0)
            s.step(5)
            outs[v] = s.get_psi()
    ref = outs[variants[0]]
    for v in variants[1:]:
        rel = np.linalg.norm(outs[v] - ref) / np.linalg.norm(ref)
        assert rel <= 1e-6, (v, rel)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("boundary", ["neumann", "periodic"])
@pytest.mark.parametrize("n,cl", [(64, 1), (64, 2), (128, 1)])
def test_pencil_tiles_are_bitwise_identical(prec, boundary, n, cl):
    """The pencil tile (lines per CTA) only regroups the lines: every built tile
    gives the default's state bit for bit, batched and advected."""
    b = 3 if n == 64 else 1
    eps = (-0.8, -0.7, -0.6)[:b]
    psi0 = S.ic.noise_batch(n, range(b), amp=0.3)
    outs = {}
    for tile in (0, 8, 16, 32):
        p = S.Params(n=n, batch=b, boundary=boundary, precision=prec, variant=cl, pencil_tile=tile,
                     eps_per_replica=eps if b > 1 else None)
        with S.Solver(p) as s:
            s.set_psi(psi0)
            s.step(20)
            outs[tile] = s.get_psi()
    for tile in (8, 16, 32):
        assert np.array_equal(outs[tile], outs[0]), tile
    pa = dict(n=n, boundary=boundary, precision=prec, advection=True, variant=cl)
    adv = {}
    for tile in (0, 8, 32):
        with S.Solver(S.Params(pencil_tile=tile, **pa)) as s:
            s.set_psi(psi0[0])
            s.step(3)
            adv[tile] = s.get_psi()
    for tile in (8, 32):
        assert np.array_equal(adv[tile], adv[0]), ("advected", tile)

