"""Autotuner for the kernel shapes of a run.

Each built shape offers a few cluster sizes for the plane pass (``variant``):
- CL = 1 and 2 at 64^3;
- CL = 1, 2 and 4 at 128^3;
- CL = 4, 8 and 16 at 256^3.

Batched runs of small grids also choose ``replica_block``: how many replicas
advance together, 16 steps at a time, while their state stays in the 126 MB L2
(0: every replica each step).  A block whose CTAs fill the GPU in about one wave
and whose fields fit L2 wins.

At 64^3, and at 128^3 with cluster size 1, the pencil pass is also built with
tiles of 8, 16 and 32 lines per CTA (``pencil_tile``): smaller tiles mean more,
smaller CTAs.

The tuner times a few steps of every built candidate for a given (n, batch,
boundary, precision, advection), first the cluster size, then the replica
block with that cluster size, then the pencil tile with both, and keeps the
fastest. Results are cached in a
JSON file keyed by that tuple and by the GPU name, under
$SMECTIC_B200_CACHE (default ~/.cache/smectic3d_b200/tuned.json).
"""
from __future__ import annotations

import dataclasses
import json
import os
import time
from pathlib import Path

import numpy as np

CANDIDATES = {16: (1,), 32: (1,), 64: (1, 2), 128: (1, 2, 4), 256: (4, 8, 16), 512: (16,)}
# replicas per L2-resident block, tried for batched plain runs at n <= 128
BLOCKS = (4, 8, 12, 13, 16, 21, 32)
# pencil tiles (lines per CTA) built besides the default
TILES = {64: (8, 16, 32), 128: (8, 16, 32)}


def cache_path() -> Path:
    base = os.environ.get("SMECTIC_B200_CACHE")
    if base:
        return Path(base)
    return Path.home() / ".cache" / "smectic3d_b200" / "tuned.json"


def _key(p, gpu: str) -> str:
    return f"{gpu}|n={p.n}|b={p.batch}|{p.boundary}|{p.precision}|adv={int(bool(p.advection))}"


def _gpu_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name(0)
    except Exception:
        return "unknown"


def _time_variant(p, variant: int, steps: int) -> float:
    from .solver import Solver
    q = dataclasses.replace(p, variant=variant, energy_trace=False, l1_interval=0)
    with Solver(q) as s:
        shape = (q.batch, q.n, q.n, q.n) if q.batch > 1 else (q.n, q.n, q.n)
        s.set_psi(np.random.default_rng(0).uniform(-0.1, 0.1, size=shape))
        s.step(2)
        s.synchronize()
        t0 = time.perf_counter()
        s.step(steps)
        t1 = time.perf_counter()
    return (t1 - t0) / steps


def tune(p, steps: int = 32, use_cache: bool = True) -> dict:
    """Time every built cluster size of ``p``'s shape, then (batched plain runs)
    every replica block with the best one; returns {"variant": best,
    "us_per_step": {variant: us}, "replica_block": b, "us_per_step_by_block":
    {b: us}} and caches it."""
    gpu = _gpu_name()
    key = _key(p, gpu)
    path = cache_path()
    cache = {}
    if path.exists():
        try:
            cache = json.loads(path.read_text())
        except ValueError:
            cache = {}
    if use_cache and key in cache:
        return cache[key]
    times = {}
    for v in CANDIDATES.get(p.n, (0,)):
        try:
            times[v] = _time_variant(p, v, steps) * 1e6
        except Exception:  # not built for this precision / shared memory
            continue
    if not times:
        raise RuntimeError(f"no plane-pass variant runs for {key}")
    best = min(times, key=times.get)
    rec = {"variant": best, "us_per_step": {str(k): v for k, v in times.items()}, "replica_block": 0}
    blocks = [b for b in BLOCKS if b < p.batch] if p.batch > 1 and p.n <= 128 and not p.advection else []
    if blocks:
        bt = {0: times[best]}
        for b in blocks:
            try:
                bt[b] = _time_variant(dataclasses.replace(p, replica_block=b), best, steps) * 1e6
            except Exception:
                continue
        rec["replica_block"] = min(bt, key=bt.get)
        rec["us_per_step_by_block"] = {str(k): v for k, v in bt.items()}
    rec["pencil_tile"] = 0
    tiles = TILES.get(p.n, ())
    if tiles:
        blk = rec["replica_block"]
        tt = {0: rec.get("us_per_step_by_block", {}).get(str(blk), times[best])}
        for tk in tiles:
            try:
                tt[tk] = _time_variant(dataclasses.replace(p, replica_block=blk, pencil_tile=tk), best, steps) * 1e6
            except Exception:  # the default tile again, or not built
                continue
        rec["pencil_tile"] = min(tt, key=tt.get)
        rec["us_per_step_by_tile"] = {str(k): v for k, v in tt.items()}
    cache[key] = rec
    path.parent.mkdir(parents=True, exist_ok=True)
    path.write_text(json.dumps(cache, indent=1, sort_keys=True))
    return rec


def best_variant(p) -> int:
    return int(tune(p)["variant"])


def best_config(p) -> tuple[int, int]:
    """(variant, replica_block) of the fastest tuned configuration."""
    rec = tune(p)
    return int(rec["variant"]), int(rec.get("replica_block", 0))


def best_shape(p) -> dict:
    """Params fields of the fastest tuned configuration: variant, replica_block,
    pencil_tile."""
    rec = tune(p)
    return {"variant": int(rec["variant"]), "replica_block": int(rec.get("replica_block", 0)),
            "pencil_tile": int(rec.get("pencil_tile", 0))}
