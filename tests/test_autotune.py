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
