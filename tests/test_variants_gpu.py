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
