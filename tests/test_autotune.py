"""Host logic of the launch-shape autotuner (no GPU): the cache key separates
table layouts, the tuner's configurations keep the caller's layout flags, and
the fastest shape is the one cached."""
import json

import torch

from poggers_b200 import autotune as at


def test_cache_key_separates_layouts(pg):
    a = pg.data_structs.hash_table_64(1 << 20, bucket=8)
    b = pg.data_structs.hash_table_64(1 << 20, bucket=8)
    b.fingerprints = True
    c = pg.data_structs.hash_table_64(1 << 21, bucket=8)
    keys = {at.cache_key("B200", x) for x in (a, b, c)}
    assert len(keys) == 3


def test_tuner_keeps_layout_flags_and_caches_the_best(pg, tmp_path, monkeypatch):
    monkeypatch.setattr(at, "CACHE", tmp_path / "tune.json")
    monkeypatch.setattr(torch.cuda, "get_device_name", lambda *a: "B200")
    cfg = pg.data_structs.hash_table_64(1 << 16, bucket=8)
    cfg.fingerprints = True
    seen = {}

    def fake_sweep(make, seed, keys, vals, qkeys, **grid):
        c = make(2, None)
        seen["fp"], seen["tile"], seen["bucket"] = c.fingerprints, c.tile, c.levels[0].bucket_size
        return [at.Result(at.Shape(t, 256, 8, 8), insert_ms=1.0 + t, query_ms=1.0) for t in (1, 2, 4)]

    monkeypatch.setattr(at, "sweep", fake_sweep)
    s = at.tuned_shape(cfg, 7, None, None, None)
    assert seen == {"fp": True, "tile": 2, "bucket": 8}
    assert s == at.Shape(1, 256, 8, 8)
    d = json.loads((tmp_path / "tune.json").read_text())
    assert list(d.values())[0]["shape"]["tile"] == 1


def test_batch_pick_is_the_fastest_shape_with_few_failures():
    R, S = at.BatchResult, at.BatchShape
    res = [R(S(1, 16, 8), 10.0, 0), R(S(1, 8, 8), 5.0, 500), R(S(2, 16, 8), 9.0, 10), R(S(4, 32, 4), 12.0, 0)]
    # the 5 ms shape fails 500 keys, far more than the fewest (0): not eligible
    assert at.best_batch(res).shape == S(2, 16, 8)


def test_batch_cache_key_separates_size_classes(pg):
    small = [pg.data_structs.tcf(1 << 12, 64) for _ in range(8)]
    large = [pg.data_structs.tcf(1 << 20, 1 << 13) for _ in range(8)]
    many = [pg.data_structs.tcf(1 << 12, 64) for _ in range(1024)]
    keys = {at.batch_cache_key("B200", c) for c in (small, large, many)}
    assert len(keys) == 3


def test_tuned_batch_shape_caches_the_pick(pg, tmp_path, monkeypatch):
    monkeypatch.setattr(at, "CACHE", tmp_path / "tune.json")
    monkeypatch.setattr(torch.cuda, "get_device_name", lambda *a: "B200")
    calls = []

    def fake_sweep(make, seeds, *a, **grid):
        calls.append(make(8)[0].levels[0].bucket_size)
        return [at.BatchResult(at.BatchShape(l, 16, 8), 1.0 + l, 0) for l in (1, 2, 4)]

    monkeypatch.setattr(at, "sweep_batch", fake_sweep)
    make = lambda b: [pg.data_structs.tcf(1 << 14, 164, bucket=b)]
    s, res = at.tuned_batch_shape(make, [1], None, None, None, None, None, None)
    assert s == at.BatchShape(1, 16, 8) and len(res) == 3 and calls == [8]
    s2, res2 = at.tuned_batch_shape(make, [1], None, None, None, None, None, None)
    assert s2 == s and res2 is None and calls == [8]
