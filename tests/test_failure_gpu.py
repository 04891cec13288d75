"""Failure detection on the GPU without a fault: every wait of the plane pass on
a cluster exchange is bounded (about 1 s), after which the kernel records a
timeout and finishes, and the call reports SH_ETIMEOUT.  The test hook
SMECTIC_B200_TEST_DROP_EXCHANGE=1 (read at sh_create) makes cluster rank 0 send
nothing in the first exchange, so its waits and its peers' expire.  A second
hook, SMECTIC_B200_TEST_FAIL_ALLOC=k, fails the k-th device allocation of
sh_create as out of memory."""
import numpy as np
import pytest

import smectic3d_b200 as S
from smectic3d_b200 import _lib as L

pytestmark = pytest.mark.gpu


def test_exchange_timeout_is_reported_and_the_context_survives(monkeypatch):
    p = S.Params(n=64, variant=2, precision="fp32")  # 64^3 with clusters of 2 CTAs
    monkeypatch.setenv("SMECTIC_B200_TEST_DROP_EXCHANGE", "1")
    with S.Solver(p) as s:
        s.set_psi(S.ic.noise(64, 0))
        with pytest.raises(S.ShError) as e:
            s.step(1)
        assert e.value.code == L.SH_ETIMEOUT
    monkeypatch.delenv("SMECTIC_B200_TEST_DROP_EXCHANGE")
    # a fresh handle on the same context steps normally
    with S.Solver(p) as s:
        s.set_psi(S.ic.noise(64, 0))
        s.step(3)
        assert np.isfinite(s.get_psi()).all()


def test_allocation_failure_is_reported_without_leaks(monkeypatch):
    """SMECTIC_B200_TEST_FAIL_ALLOC=k makes the k-th device allocation of sh_create
    fail as out of memory: the call returns SH_ENOMEM, frees what it had allocated
    (free device memory is unchanged after many such calls) and later handles work."""
    import torch
    p = S.Params(n=256, precision="fp32")
    for k in (1, 3, 5, 7):
        monkeypatch.setenv("SMECTIC_B200_TEST_FAIL_ALLOC", str(k))
        with pytest.raises(S.ShError) as e:
            S.Solver(p)
        assert e.value.code == L.SH_ENOMEM
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(20):
        with pytest.raises(S.ShError):
            S.Solver(p)
    torch.cuda.synchronize()
    assert free0 - torch.cuda.mem_get_info()[0] < 64 * 2**20
    monkeypatch.delenv("SMECTIC_B200_TEST_FAIL_ALLOC")
    with S.Solver(S.Params(n=64, precision="fp32")) as s:
        s.set_psi(S.ic.noise(64, 0))
        s.step(2)
        assert np.isfinite(s.get_psi()).all()
