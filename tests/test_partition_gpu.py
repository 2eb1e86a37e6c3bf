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


def _few_buckets(keys, seed=43, nslots=NSLOTS, bucket=8):
    """Keys whose 20 double-hash probes cover at most two distinct buckets (the
    second hash a multiple of nb / 2 when nb is a power of two): whether they
    fit depends on placement order, in the reference as well."""
    from oracle import pyoracle
    nb = nslots // bucket
    return np.array([len({v % nb for v in pyoracle.probe_values(0, seed, 0, int(k), 20)}) <= 2 for k in keys],
                    dtype=bool)


def test_ordered_insert_without_values_and_flags(pg):
    import torch
    n = 3 << 20
    keys = wl.keys_without_sentinels(7, n)
    t = _table(pg, "interleaved", True)
    fails = torch.zeros(1, dtype=torch.int64, device="cuda")
    t.bulk_insert(to_dev(keys), None, None, fails)  # NULL values and NULL flags
    torch.cuda.synchronize()
    f, v = Driver(t).query(keys)
    assert int(fails.item()) == int((~f).sum()) and _few_buckets(keys[~f]).all()
    assert (v == 0).all()
    # a second, smaller ordered batch reuses the scratch
    before = t.host_bytes_in_use()
    more = wl.keys_without_sentinels(8, 1 << 20)
    ok = Driver(t).insert(more, wl.values_for(more, 8, 5))
    assert _few_buckets(more[~ok]).all() and t.host_bytes_in_use() == before


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
def test_bucketed_filter_keeps_batch_order(pg, bits):
    """The bucketed filter is never region-sorted: with region ordering on, a
    large insert at 0.9 load allocates no scratch and sends as many keys to the
    1 % backing level as with it off.  (Sorting by the first choice would
    unbalance the two choices, about 5x the keys reaching the backing level,
    and would change which keys the linear level displaces, which its
    live-fill stop rule makes visible to later removes.)"""
    from tests.test_bucketed_gpu import _run
    n0 = 1 << 25 if bits == 16 else 1 << 26
    n = int(0.9 * n0)
    keys = wl.keys_without_sentinels(73, n)
    vals = wl.values_for(keys, 2, 74).astype(np.uint64) & np.uint64((1 << bits) - 1)
    backing = []
    for part in (True, False):
        t = pg.Table(pg.data_structs.del_tcf(n0, n0 // 100, tag_bits=bits), 5)
        t.set_partitioned_insert(part)
        before = t.host_bytes_in_use()
        ok, _, _ = _run(pg, t, bits, 0, keys, vals)
        _run(pg, t, bits, 2, keys[:1 << 21])
        a, _, _ = _run(pg, t, bits, 3, keys[:1 << 21], vals[:1 << 21])
        assert ok.all() and a.all() and t.host_bytes_in_use() == before
        backing.append(t.get_fill(1)[0])
        t.free_on_device()
    assert abs(backing[0] - backing[1]) <= max(500, backing[1] // 10), backing


def test_ordered_insert_with_a_full_run(pg):
    """A batch far from uniform over the table: 2^19 copies of one key on top of
    2^21 distinct keys.  The copies overflow their region's run; those that do
    not fit are inserted by the second pass in batch order.  Both runs (sorted
    and batch order) place every distinct key (but those whose probes cover at
    most two buckets), fill most of the copies' 20 buckets (at most 20 probes x
    8 slots) and report each failure at its own batch position."""
    uniq = wl.keys_without_sentinels(15, 1 << 21)
    dup = np.full(1 << 19, uniq[0], dtype=np.uint64)
    keys = np.concatenate([uniq[: 1 << 20], dup, uniq[1 << 20:]])
    vals = wl.values_for(keys, 8, 16)
    is_dup = np.zeros(len(keys), dtype=bool)
    is_dup[1 << 20: (1 << 20) + (1 << 19)] = True
    is_dup[0] = True  # the first copy of the key is uniq[0] itself
    placed = []
    for part in (True, False):
        t = _table(pg, "fingerprints", part)
        d = Driver(t)
        ok = d.insert(keys, vals)
        assert _few_buckets(keys[~is_dup & ~ok]).all()
        f, v = d.query(uniq[1:])
        assert (f == ok[~is_dup]).all() and (v[f] == vals[~is_dup][f]).all()
        placed.append(int(ok[is_dup].sum()))
        assert t.get_fill(0)[0] == int(ok.sum())
        t.free_on_device()
    # the copies fill the key's 20 buckets (160 slots) but for the distinct keys
    # that concurrent placement put there first, which differs between the runs
    assert all(100 <= p <= 160 for p in placed) and abs(placed[0] - placed[1]) <= 32, placed


def test_reserved_scratch_means_no_allocation_in_the_insert(pg):
    """pg_table_reserve_insert_scratch grows the region sort's scratch ahead
    of time: a region-ordered insert of that size then adds nothing to the
    table's device bytes, and every key is found with its value."""
    import torch
    from tests.gpu_util import Driver
    cfg = pg.data_structs.hash_table_64(1 << 23, bucket=8)
    cfg.fingerprints = True
    t = pg.Table(cfg, 12)
    n = 1 << 21
    before = t.host_bytes_in_use()
    t.reserve_insert_scratch(n)
    torch.cuda.synchronize()
    reserved = t.host_bytes_in_use()
    assert reserved > before
    keys = wl.keys_without_sentinels(13, n)
    vals = wl.values_for(keys, 8, 14)
    ok = Driver(t).insert(keys, vals)
    assert t.host_bytes_in_use() == reserved and ok.all()
    f, v = Driver(t).query(keys)
    assert f.all() and (v == vals).all()


def test_wide_tile_scatter_for_many_regions(pg):
    """A table of more than 64 regions (2^28 slots, 4 GiB: 128 regions) sorts
    with the wide-tile scatter.  The batch holds 0.8 x 2^28 distinct keys and
    2^20 copies of one key between them, so that key's run overflows and the
    second pass takes the rest.  The bucket rule allows a key to fail only when
    every bucket of its probe sequence is full: checked on a dump of the level
    for each failed key (a handful: region order fills a region's buckets
    before the next region's keys probe into it) and for the copied key, whose
    copies beyond its buckets' 160 slots must fail.  Every placed key is found
    with its own value, flagged at its own batch position, and the level's
    fill equals the keys placed."""
    import ctypes
    import torch
    from oracle import pyoracle
    ns = 1 << 28
    nb = ns // 8
    nu = int(0.8 * ns)
    ndup = 1 << 20
    cfg = pg.data_structs.hash_table_64(ns, bucket=8)
    cfg.fingerprints = True
    t = pg.Table(cfg, 44)
    uniq = wl.device_splitmix64(61, nu)
    dup_key = uniq[:1]
    keys = torch.cat([uniq[: nu // 2], dup_key.expand(ndup), uniq[nu // 2:]])
    vals = wl.device_splitmix64(62, nu + ndup)
    ok = torch.zeros(nu + ndup, dtype=torch.uint8, device="cuda")
    t.bulk_insert(keys, vals, ok)
    is_dup = torch.zeros(nu + ndup, dtype=torch.bool, device="cuda")
    is_dup[nu // 2: nu // 2 + ndup] = True
    is_dup[0] = True  # uniq[0] is the duplicated key
    okb = ok.bool()
    failed = keys[~is_dup & ~okb].cpu().numpy().view(np.uint64)
    assert len(failed) < 100, len(failed)
    placed_dups = int(okb[is_dup].sum().item())
    assert 0 < placed_dups <= 160, placed_dups
    assert t.get_fill(0)[0] == int(okb.sum().item())
    # a failed key's probe buckets are all full (slot key 0 = empty)
    dump = np.empty(2 * ns, dtype=np.uint64)
    assert pg.lib().pg_table_dump_level(t._h, 0, ctypes.c_void_p(dump.ctypes.data), dump.nbytes) == 0
    slot_keys = dump[0::2]
    for k in list(failed) + [int(uniq[0].item()) & ((1 << 64) - 1)]:
        for b in {v % nb for v in pyoracle.probe_values(0, 44, 0, int(k), 20)}:
            assert (slot_keys[8 * b: 8 * b + 8] != 0).all(), (k, b)
    del dump, slot_keys
    q = uniq[1:]
    found = torch.zeros(nu - 1, dtype=torch.uint8, device="cuda")
    qv = torch.zeros(nu - 1, dtype=torch.int64, device="cuda")
    t.bulk_query(q, qv, found)
    exp_ok = okb[~is_dup]
    exp_v = vals[~is_dup]
    assert torch.equal(found.bool(), exp_ok)
    assert torch.equal(qv[exp_ok], exp_v[exp_ok])
    t.free_on_device()
