"""Host-side logic of the multi-GPU mode (replicas only), on two gloo ranks on
CPU: every rank integrates its own domain, the job time is the slowest rank's
and the throughput counts the steps of all ranks."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms_local = 10.0 * (rank + 1)            # rank 1 is the slow one
        rate, ms = bench.aggregate_rate(100, ms_local, torch, dist, device="cpu")
        out[rank] = (rate, ms)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replica_throughput_uses_slowest_rank():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    for r in range(world):
        rate, ms = out[r]
        assert ms == pytest.approx(20.0)
        assert rate == pytest.approx(world * 100 / 0.020)


def _inputs_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p, psi0 = bench.rank_inputs("periodic128", rank)
        mine = torch.tensor([float(psi0.sum()), float((psi0 * psi0).sum())], dtype=torch.float64)
        got = [torch.zeros(2, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(got, mine)
        out[rank] = ([g.tolist() for g in got], p.n, p.batch)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_ranks_integrate_distinct_seeded_domains():
    """bench.run_ours' inputs on two gloo ranks: each rank seeds its own domain
    by its rank, so the domains differ and each is reproducible."""
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_inputs_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    sums = out[0][0]
    assert out[1][0] == sums  # every rank sees the same gathered checksums
    assert sums[0] != sums[1]
    for r in range(world):
        _, psi = bench.rank_inputs("periodic128", r)
        assert [float(psi.sum()), float((psi * psi).sum())] == pytest.approx(sums[r], rel=1e-15)
        assert out[r][1:] == (128, 1)


def test_single_rank_passthrough():
    rate, ms = bench.aggregate_rate(50, 5.0, torch, None)
    assert ms == 5.0 and rate == pytest.approx(50 / 0.005)
