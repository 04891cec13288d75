"""sh_l1_noalloc, the L1 monitor that allocates no device memory, against the
handle-based monitor behind sh_l1 and against the oracle's L1 monitor.

sh_l1_noalloc is for callers that cannot let a library call cudaMalloc:
 - hosts that own all device memory through their own pool;
 - real-time loops that cannot take the implicit synchronisation of an
   allocation.
This test therefore owns every device buffer it passes. It checks the result
against the value sh_l1 reports for the same two states and against the
oracle's monitor evaluated on copies of those states, on two calls in a row.
The second call must not see anything the first one left in the shared
scratch array.
"""
import numpy as np
import pytest

import smectic3d_b200 as S
from oracle import sh_oracle as O
from smectic3d_b200 import _lib as L

pytestmark = pytest.mark.gpu


def test_l1_noalloc_matches_handle_monitor_twice():
    import torch

    n, batch, k = 32, 2, 5
    p = S.Params(n=n, batch=batch, precision="fp64", l1_interval=k, eps_per_replica=(-0.8, -0.6))
    lib = L.load()
    psi0 = S.ic.noise_batch(n, (1, 2), 0.4) + 1.3 * np.cos(np.arange(n) * p.dx)[None, None, None, :]
    size = batch * n ** 3
    old = torch.empty(size, dtype=torch.float64, device="cuda")
    new = torch.empty(size, dtype=torch.float64, device="cuda")
    out = torch.empty(batch, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    with S.Solver(p) as s:
        s.set_psi(psi0)
        for call in range(2):
            s.step(k - 1)
            s.get_psi_device(old.data_ptr())
            s.step(1)
            s.get_psi_device(new.data_ptr())
            ref, cnt = s.l1()
            assert cnt == call + 1
            out.fill_(float("nan"))
            torch.cuda.synchronize()
            rc = lib.sh_l1_noalloc(new.data_ptr(), old.data_ptr(), n ** 3, batch, p.dt, out.data_ptr(), s.stream)
            assert rc == L.SH_OK, lib.sh_last_error(None)
            s.synchronize()
            got = out.cpu().numpy()
            assert np.all(np.isfinite(got))
            assert np.allclose(got, ref, rtol=1e-12, atol=0), (call, got, ref)
            a_new = new.cpu().numpy().reshape(batch, -1)
            a_old = old.cpu().numpy().reshape(batch, -1)
            orc = [O.l1_monitor(a_new[r], a_old[r], p.dt) for r in range(batch)]
            assert np.allclose(got, orc, rtol=1e-12, atol=0), (call, got, orc)


def test_l1_noalloc_rejects_batch_beyond_scratch():
    lib = L.load()
    buf = 0x1000  # never dereferenced: the size check comes first
    rc = lib.sh_l1_noalloc(buf, buf, 8, 129, 0.05, buf, None)
    assert rc == L.SH_EINVAL
    assert b"128" in lib.sh_last_error(None)
