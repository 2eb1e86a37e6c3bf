"""GPU tests of region-ordered inserts (large batches into large uint64 tables).

The insert kernel visits a counting-sorted copy of the batch; the per-key rule
is unchanged.  Bar: every key that both an ordered and an unordered run placed
answers queries identically (and identically to the oracle), each run agrees
with its own insert report, and the ok flags land at the caller's positions.
"""
import numpy as np
import pytest

from tests.gpu_util import Driver, to_dev
from poggers_b200 import workload as wl

pytestmark = pytest.mark.gpu

NSLOTS = 1 << 23  # 128 MB of uint64 slots: 4 regions of 32 MB


def _table(pg, layout, partition, nslots=NSLOTS, bucket=8):
    cfg = pg.data_structs.hash_table_64(nslots, bucket=bucket)
    cfg.split = layout == "split"
    cfg.fingerprints = layout == "fingerprints"
    t = pg.Table(cfg, 43)
    t.set_partitioned_insert(partition)
    return t


@pytest.mark.parametrize("layout", ["interleaved", "split", "fingerprints"])
def test_ordered_insert_matches_unordered_and_oracle(pg, oracle, layout):
    n = int(0.9 * NSLOTS)
    keys = wl.keys_without_sentinels(43, n)
    vals = wl.values_for(keys, 8, 50)
    half = n // 2
    q = np.concatenate([keys[:half], wl.keys_without_sentinels(4343, half)])
    a, b = _table(pg, layout, True), _table(pg, layout, False)
    da, db = Driver(a), Driver(b)
    oka, okb = da.insert(keys, vals), db.insert(keys, vals)
    assert (~oka).sum() < 200 and (~okb).sum() < 200
    assert a.host_bytes_in_use() > b.host_bytes_in_use()  # the sort's scratch is the table's
    fa, va = da.query(q)
    fb, vb = db.query(q)
    # each run agrees with its own insert report
    assert (fa[:half] == oka[:half]).all() and (fb[:half] == okb[:half]).all()
    assert (va[:half][oka[:half]] == vals[:half][oka[:half]]).all()
    both = np.concatenate([oka[:half] & okb[:half], np.ones(half, dtype=bool)])
    assert (fa[both] == fb[both]).all() and (va[both] == vb[both]).all()
    o = oracle.OracleTable(0, 4, [(NSLOTS, 8, 20, 0, 0)], 43)
    oko = o.insert_many(keys, vals, threads=8)
    fo, vo = o.query_many(q, threads=8)
    both &= np.concatenate([oko[:half], np.ones(half, dtype=bool)])
    assert (fa[both] == fo[both]).all() and (va[both] == vo[both]).all()
    # removes after an ordered insert
    ridx = wl.fisher_yates_half(n, 77)
    r = da.remove(keys[ridx])
    assert (r == oka[ridx]).all()


def test_ordered_insert_without_values_and_flags(pg):
    import torch
    n = 3 << 20
    keys = wl.keys_without_sentinels(7, n)
    t = _table(pg, "interleaved", True)
    fails = torch.zeros(1, dtype=torch.int64, device="cuda")
    t.bulk_insert(to_dev(keys), None, None, fails)  # NULL values and NULL flags
    torch.cuda.synchronize()
    assert int(fails.item()) == 0
    f, v = Driver(t).query(keys)
    assert f.all() and (v == 0).all()
    # a second, smaller ordered batch reuses the scratch
    before = t.host_bytes_in_use()
    more = wl.keys_without_sentinels(8, 1 << 20)
    ok = Driver(t).insert(more, wl.values_for(more, 8, 5))
    assert ok.all() and t.host_bytes_in_use() == before


def test_ordered_insert_overflow_reports_each_failure_in_place(pg):
    """A table too small for the batch: the failures that the run reports are
    exactly the keys that queries do not find, at their own batch positions."""
    nslots = 1 << 22  # 64 MB: 2 regions
    n = nslots + (nslots >> 3)
    keys = wl.keys_without_sentinels(99, n)
    vals = wl.values_for(keys, 8, 3)
    t = _table(pg, "interleaved", True, nslots=nslots)
    d = Driver(t)
    ok = d.insert(keys, vals)
    assert (~ok).sum() >= n - nslots
    f, v = d.query(keys)
    assert (f == ok).all()
    assert (v[ok] == vals[ok]).all()


def test_small_batches_take_the_unordered_path(pg):
    t = _table(pg, "interleaved", True)
    keys = wl.keys_without_sentinels(5, (1 << 20) - 1)
    ok = Driver(t).insert(keys, wl.values_for(keys, 8, 1))
    assert ok.all()
    b = _table(pg, "interleaved", False)
    assert t.host_bytes_in_use() == b.host_bytes_in_use()


@pytest.mark.parametrize("bits", [16, 8])
def test_ordered_insert_of_bucketed_filter(pg, bits):
    """The bucketed filter's insert and insert_with_delete on a region-sorted
    batch (a 2^25-slot primary level: 128 MiB at 16-bit tags): every key
    placed, found, its flag at its own batch position; fills equal the
    unordered run's; re-adds through insert_with_delete likewise."""
    from tests.test_bucketed_gpu import _run
    n0 = 1 << 25 if bits == 16 else 1 << 26
    n1 = n0 // 100
    n = 3 << 20
    keys = wl.keys_without_sentinels(71, n)
    mask = (1 << bits) - 1
    vals = wl.values_for(keys, 2, 72).astype(np.uint64) & np.uint64(mask)
    runs = []
    for part in (True, False):
        t = pg.Table(pg.data_structs.del_tcf(n0, n1, tag_bits=bits), 5)
        t.set_partitioned_insert(part)
        ok, _, _ = _run(pg, t, bits, 0, keys, vals)
        f, v, _ = _run(pg, t, bits, 1, keys)
        r, _, _ = _run(pg, t, bits, 2, keys[: n // 2])
        a, _, _ = _run(pg, t, bits, 3, keys[: n // 2], vals[: n // 2])
        fills = [t.get_fill(0), t.get_fill(1)]
        runs.append((ok, f, v, r, a, fills, t.host_bytes_in_use()))
    (ok1, f1, v1, r1, a1, fl1, b1), (ok2, f2, v2, r2, a2, fl2, b2) = runs
    assert ok1.all() and ok2.all() and f1.all() and f2.all() and a1.all() and a2.all()
    assert b1 > b2  # the sort's scratch belongs to the table
    def live(fl):
        return sum(o - t for o, t in fl)
    assert live(fl1) == n - int(r1.sum()) + int(a1.sum())
    assert live(fl2) == n - int(r2.sum()) + int(a2.sum())
    assert abs(int(r1.sum()) - int(r2.sum())) <= 10
    # a shared tag answers with the value of whichever key holds the earlier slot:
    # both orders show the same collision rate
    m1, m2 = (v1 != vals).mean(), (v2 != vals).mean()
    if bits == 16:
        assert m1 < 0.001 and m2 < 0.001
    else:
        assert abs(m1 - m2) <= 0.2 * max(m1, m2) + 0.001
