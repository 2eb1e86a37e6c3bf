"""GPU tests of checkpoint images: save a table, restore it (also from a
file), and find the same bytes and the same answers."""
import numpy as np
import pytest

from tests.gpu_util import Driver
from poggers_b200 import workload as wl

pytestmark = pytest.mark.gpu


def _configs(pg):
    fp = pg.data_structs.hash_table_64(1 << 14, bucket=8)
    fp.fingerprints = True
    sp = pg.data_structs.hash_table_64(1 << 14, bucket=8)
    sp.split = True
    return {
        "ht": pg.data_structs.hash_table_64(1 << 14, bucket=8),
        "ht_fingerprints": fp,
        "ht_split": sp,
        "tcf": pg.data_structs.tcf(1 << 14, 1 << 8),
        "del_tcf": pg.data_structs.del_tcf(1 << 14, 1 << 8),
    }


@pytest.mark.parametrize("name", ["ht", "ht_fingerprints", "ht_split", "tcf", "del_tcf"])
def test_image_round_trip(pg, tmp_path, name):
    cfg = _configs(pg)[name]
    t = pg.Table(cfg, 77)
    d = Driver(t)
    keys = wl.keys_without_sentinels(5, 12000)
    vbytes = 8 if cfg.format == pg.FMT_KV64 else 2
    vals = wl.values_for(keys, vbytes, 6).astype(np.uint64)
    if cfg.format != pg.FMT_KV64:
        vals &= np.uint64(0xFFFF)
    ok = d.insert(keys, vals)
    d.remove(keys[:3000])
    q = np.concatenate([keys, wl.keys_without_sentinels(9, 3000)])
    f0, v0 = d.query(q)
    path = tmp_path / f"{name}.pgimg"
    t.save(path)
    u = pg.Table.load(path)
    assert u.config.format == cfg.format and u.seed == 77
    for lv in range(len(cfg.levels)):
        assert u.dump_level(lv) == t.dump_level(lv)
    f1, v1 = Driver(u).query(q)
    assert (f0 == f1).all() and (v0 == v1).all()
    assert ok.sum() > 11000


def test_corrupt_image_is_refused(pg):
    t = pg.Table(pg.data_structs.hash_table_64(1 << 10, bucket=8), 3)
    img = bytearray(t.save_image())
    img[200] ^= 0x40
    with pytest.raises(pg.PoggersError):
        pg.Table.from_image(bytes(img))
