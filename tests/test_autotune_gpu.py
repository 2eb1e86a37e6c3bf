"""GPU test of the launch-shape autotuner: a small sweep returns a shape of
the grid, the result is cached per GPU and table shape, and a cached shape is
returned without sweeping again."""
import pytest

from tests.gpu_util import to_dev
from poggers_b200 import workload as wl

pytestmark = pytest.mark.gpu


def test_tuned_shape_sweeps_once_then_uses_the_cache(pg, tmp_path, monkeypatch):
    from poggers_b200 import autotune as at
    monkeypatch.setattr(at, "CACHE", tmp_path / "tune.json")
    cfg = pg.data_structs.hash_table_64(1 << 15, bucket=8)
    keys = wl.keys_without_sentinels(3, 25000)
    q = wl.keys_without_sentinels(4, 25000)
    k, v, qk = to_dev(keys), to_dev(wl.values_for(keys, 8, 5)), to_dev(q)
    grid = dict(tiles=(1, 2), block_threads=(256,), blocks_per_sm=(8,), reps=1)
    s1 = at.tuned_shape(cfg, 7, k, v, qk, **grid)
    assert s1.tile in (1, 2) and s1.block_threads == 256 and s1.bucket == 8
    assert (tmp_path / "tune.json").exists()

    def no_sweep(*a, **kw):
        raise AssertionError("the cached shape should have been used")

    monkeypatch.setattr(at, "sweep", no_sweep)
    assert at.tuned_shape(cfg, 7, k, v, qk, **grid) == s1
    # a fingerprinted table is a different shape of table: a cache miss
    fcfg = pg.data_structs.hash_table_64(1 << 15, bucket=8)
    fcfg.fingerprints = True
    with pytest.raises(AssertionError):
        at.tuned_shape(fcfg, 7, k, v, qk, **grid)
