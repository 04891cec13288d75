"""Host logic of the cluster-size autotuner (no GPU): the fastest built
variant wins, variants that fail to build are skipped, results are cached per
(GPU, shape) and reused."""
import json

import pytest

import smectic3d_b200 as S
from smectic3d_b200 import autotune


@pytest.fixture
def fake(monkeypatch, tmp_path):
    cache = tmp_path / "tuned.json"
    monkeypatch.setenv("SMECTIC_B200_CACHE", str(cache))
    monkeypatch.setattr(autotune, "_gpu_name", lambda: "FakeGPU")
    calls = []

    def timer(us):
        def _time_variant(p, v, steps):
            calls.append(v)
            if us[v] is None:
                raise RuntimeError("variant not built")
            return us[v] * 1e-6
        return _time_variant
    return cache, calls, timer


def test_fastest_variant_wins_and_is_cached(fake, monkeypatch):
    cache, calls, timer = fake
    monkeypatch.setattr(autotune, "_time_variant", timer({4: 250.0, 8: 200.0, 16: 210.0}))
    p = S.Params(n=256, boundary="neumann", precision="fp32")
    rec = autotune.tune(p, steps=3)
    assert rec["variant"] == 8
    assert set(rec["us_per_step"]) == {"4", "8", "16"}
    assert calls == [4, 8, 16]
    stored = json.loads(cache.read_text())
    assert list(stored) == ["FakeGPU|n=256|b=1|neumann|fp32|adv=0"]
    # a second call reads the cache and times nothing
    assert autotune.tune(p, steps=3) == rec and calls == [4, 8, 16]
    assert autotune.best_variant(p) == 8
    # use_cache=False times again
    autotune.tune(p, steps=3, use_cache=False)
    assert calls == [4, 8, 16, 4, 8, 16]


def test_unbuilt_variants_are_skipped(fake, monkeypatch):
    _, _, timer = fake
    monkeypatch.setattr(autotune, "_time_variant", timer({1: 30.0, 2: None, 4: 25.0}))
    rec = autotune.tune(S.Params(n=128, precision="fp64"), steps=3)
    assert rec["variant"] == 4 and "2" not in rec["us_per_step"]


def test_no_variant_raises(fake, monkeypatch):
    _, _, timer = fake
    monkeypatch.setattr(autotune, "_time_variant", timer({1: None, 2: None}))
    with pytest.raises(RuntimeError, match="no plane-pass variant"):
        autotune.tune(S.Params(n=64, precision="fp32"), steps=3)


def test_keys_separate_shapes(fake, monkeypatch):
    cache, _, timer = fake
    monkeypatch.setattr(autotune, "_time_variant", timer({1: 10.0, 2: 5.0}))
    autotune.tune(S.Params(n=64, precision="fp32", batch=8), steps=3)
    autotune.tune(S.Params(n=64, precision="fp32", batch=8, boundary="neumann"), steps=3)
    assert len(json.loads(cache.read_text())) == 2


def test_replica_block_is_tuned_for_batched_runs(fake, monkeypatch):
    """Batched plain runs then try replica blocks below the batch with the best
    cluster size; the fastest (or no blocking) is kept."""
    cache, calls, _ = fake
    seen = []

    def _time_variant(p, v, steps):
        seen.append((v, p.replica_block))
        base = {1: 100.0, 2: 120.0}[v]
        return (base - (40.0 if p.replica_block == 13 else 0.0)) * 1e-6
    monkeypatch.setattr(autotune, "_time_variant", _time_variant)
    rec = autotune.tune(S.Params(n=64, precision="fp32", batch=64), steps=3)
    assert rec["variant"] == 1 and rec["replica_block"] == 13
    assert seen[:2] == [(1, 0), (2, 0)]
    assert {b for v, b in seen[2:]} == {4, 8, 12, 13, 16, 21, 32} and all(v == 1 for v, _ in seen[2:])
    assert autotune.best_config(S.Params(n=64, precision="fp32", batch=64)) == (1, 13)
    # single domains and advected runs are not blocked
    seen.clear()
    rec = autotune.tune(S.Params(n=64, precision="fp32", batch=1), steps=3)
    assert rec["replica_block"] == 0 and all(b == 0 for _, b in seen)


def test_pencil_tile_is_tuned_at_64(fake, monkeypatch):
    """At 64^3 the tuner then tries the pencil tiles with the best cluster size
    and replica block; best_shape returns all three Params fields."""
    seen = []

    def _time_variant(p, v, steps):
        seen.append((v, p.replica_block, p.pencil_tile))
        return ({1: 100.0, 2: 120.0}[v] - (30.0 if p.pencil_tile == 32 else 0.0)) * 1e-6
    monkeypatch.setattr(autotune, "_time_variant", _time_variant)
    p = S.Params(n=64, precision="fp32", batch=1)
    rec = autotune.tune(p, steps=3)
    assert rec["variant"] == 1 and rec["pencil_tile"] == 32
    assert {t for _, _, t in seen[2:]} == {8, 16, 32} and all(v == 1 for v, _, _ in seen[2:])
    assert autotune.best_shape(p) == {"variant": 1, "replica_block": 0, "pencil_tile": 32}
    # sizes without tile variants keep the default
    seen.clear()
    monkeypatch.setattr(autotune, "_time_variant", lambda p, v, steps: {4: 1e-5, 8: 2e-5, 16: 3e-5}[v])
    assert autotune.tune(S.Params(n=256, precision="fp64"), steps=3)["pencil_tile"] == 0
