"""CPU tests: the oracle pinned to the reference, and oracle semantics.

The oracle's hashing and probing are checked bit for bit against the
reference's own code compiled for the host (oracle/_ref/libpoggers_refhost.so);
its table model is checked byte for byte against golden dumps recorded from
the reference's CUDA build (tests/golden/).
"""
import ctypes as C

import numpy as np
import pytest

from tests.cases import BCASES, CASES, golden, oracle_btable, oracle_table
from poggers_b200 import workload as wl


def test_splitmix_matches_numpy(oracle):
    a = oracle.splitmix64(42, 10000)
    b = wl.splitmix64(42, 10000)
    assert (a == b).all()
    assert len(np.unique(a)) == len(a)


def test_murmur_pinned_to_reference(oracle):
    rh = oracle.refhost()
    if rh is None:
        pytest.skip("reference host build absent (make -C oracle ref)")
    keys = list(map(int, wl.splitmix64(1, 3000))) + [0, 1, (1 << 64) - 1, 0x8000000000000000]
    for s in (42, 43, 42 * 42, (42 ** 4) % (1 << 64), 0, (1 << 64) - 1):
        for k in keys:
            assert oracle.murmur64a(k, s) == rh.refh_murmur64a(k, s)


@pytest.mark.parametrize("kind,maxp", [(0, 20), (1, 20), (2, 2), (3, 2)])
def test_probe_sequences_pinned_to_reference(oracle, kind, maxp):
    rh = oracle.refhost()
    if rh is None:
        pytest.skip("reference host build absent (make -C oracle ref)")
    for fmt in (0, 1):
        for k in map(int, wl.splitmix64(7 + kind, 2000)):
            tag = k if fmt == 0 else int(oracle.lib().pgo_tag16(k))
            ref = (C.c_uint64 * 32)()
            n = rh.refh_probe_values(kind, 42, k, tag, ref, 32)
            assert list(ref[:n]) == oracle.probe_values(kind, 42, fmt, k, maxp)


def test_tag16_remaps_sentinels(oracle):
    t = oracle.lib().pgo_tag16
    assert t(0) == 1 and t(0x10000) == 1
    assert t(0xFFFF) == 0xFFFE and t(0xABCD0000FFFF) == 0xFFFE
    assert t(0x1234) == 0x1234


def _replay(oracle, name, g, partition=None):
    t = oracle_table(oracle, name, partition)
    ok = t.insert_many(g["keys"], g["vals"])
    dumps = [t.level_bytes(l) for l in range(t.nlevels)]
    qf, qv = t.query_many(g["qkeys"])
    rok = t.remove_many(g["rkeys"])
    dumps2 = [t.level_bytes(l) for l in range(t.nlevels)]
    qf2, qv2 = t.query_many(g["qkeys"])
    return ok, dumps, qf, qv, rok, dumps2, qf2, qv2


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_golden(oracle, name):
    g = golden(name)
    if g is None:
        pytest.skip(f"golden fixture ref_{name}.npz not recorded yet")
    ok, dumps, qf, qv, rok, dumps2, qf2, qv2 = _replay(oracle, name, g)
    assert (ok == g["insert_ok"].astype(bool)).all()
    for l, d in enumerate(dumps):
        assert d == g[f"dump_insert_l{l}"].tobytes(), f"level {l} layout after inserts"
    assert (qf == g["q_found"].astype(bool)).all()
    assert (qv == g["q_vals"]).all()
    assert (rok == g["remove_ok"].astype(bool)).all()
    for l, d in enumerate(dumps2):
        assert d == g[f"dump_remove_l{l}"].tobytes(), f"level {l} layout after removes"
    assert (qf2 == g["q2_found"].astype(bool)).all()
    assert (qv2 == g["q2_vals"]).all()


@pytest.mark.parametrize("name", sorted(CASES))
def test_tile_width_does_not_change_results(oracle, name):
    """Filled slots form a prefix of each bucket, so the reference's stripe width
    (Partition_Size) never changes a result of phase-separated operations."""
    fmt, tile, levels, seed = CASES[name]
    keys = np.concatenate([wl.keys_without_sentinels(99, 1500), np.array([0, (1 << 64) - 1], dtype=np.uint64)])
    g = {"keys": keys, "vals": wl.values_for(keys, 8, 3).astype(np.uint64),
         "qkeys": np.concatenate([keys, wl.keys_without_sentinels(98, 300)]), "rkeys": keys[:400]}
    if fmt != 0:
        g["vals"] &= np.uint64(0xFFFF)
    base = _replay(oracle, name, g, partition=1)
    for p in (2, 4):
        other = _replay(oracle, name, g, partition=p)
        for a, b in zip(base, other):
            if isinstance(a, list):
                assert a == b
            else:
                assert (a == b).all()


def test_sentinel_semantics_ht(oracle):
    """key 0 is the empty key and ~0 the tombstone of key_val_pair<uint64,uint64>:
    inserting 0 writes a value into an empty slot without claiming it; querying 0
    reports the first empty slot; removing 0 turns an empty slot into a tombstone."""
    t = oracle.OracleTable(0, 4, [(64, 8, 20, 0, 0)], 5)
    assert t.insert_many(np.array([0], dtype=np.uint64), np.array([77], dtype=np.uint64)).all()
    assert t.count_fill(0) == 0
    f, v = t.query_many(np.array([0], dtype=np.uint64))
    assert f[0] and v[0] == 77
    assert t.remove_many(np.array([0], dtype=np.uint64)).all()
    assert t.count_fill(0) == 1
    f, v = t.query_many(np.array([0], dtype=np.uint64))
    assert f[0] and v[0] == 0  # the next empty slot of the same bucket


def test_duplicate_keys_take_two_slots_and_query_returns_first(oracle):
    t = oracle.OracleTable(0, 4, [(64, 8, 20, 0, 0)], 5)
    k = np.array([12345, 12345], dtype=np.uint64)
    assert t.insert_many(k, np.array([1, 2], dtype=np.uint64)).all()
    assert t.count_fill(0) == 2
    f, v = t.query_many(k[:1])
    assert f[0] and v[0] == 1
    assert t.remove_many(k[:1]).all()
    f, v = t.query_many(k[:1])
    assert f[0] and v[0] == 2


def test_full_table_reports_failures(oracle):
    t = oracle.OracleTable(0, 4, [(64, 8, 20, 0, 0)], 5)
    keys = wl.keys_without_sentinels(3, 200)
    ok = t.insert_many(keys)
    assert ok.sum() <= 64 and (~ok).sum() >= 136
    f, _ = t.query_many(keys)
    assert (f == ok).all()


def test_multithreaded_port_matches_sequential_ht(oracle):
    keys = wl.keys_without_sentinels(11, 90000)
    vals = wl.values_for(keys, 8, 12)
    q = np.concatenate([keys[:45000], wl.keys_without_sentinels(13, 45000)])
    seq = oracle.OracleTable(0, 4, [(100000, 8, 20, 0, 0)], 43)
    mt = oracle.OracleTable(0, 4, [(100000, 8, 20, 0, 0)], 43)
    ok_s = seq.insert_many(keys, vals)
    ok_m = mt.insert_many(keys, vals, threads=4)
    # at 0.9 load a handful of inserts fail; which ones depends on the order
    assert (~ok_s).sum() < 20 and (~ok_m).sum() < 20
    both = np.concatenate([ok_s[:45000] & ok_m[:45000], np.ones(45000, dtype=bool)])
    a = seq.query_many(q)
    b = mt.query_many(q, threads=4)
    assert (a[0][both] == b[0][both]).all() and (a[1][both] == b[1][both]).all()
    assert (b[0][:45000] == ok_m[:45000]).all()
    ridx = wl.fisher_yates_half(len(keys), 5)
    rs, rm = seq.remove_many(keys[ridx]), mt.remove_many(keys[ridx], threads=4)
    assert (rs == ok_s[ridx]).all() and (rm == ok_m[ridx]).all()
    a = seq.query_many(q)
    b = mt.query_many(q, threads=4)
    assert (a[0][both] == b[0][both]).all() and (a[1][both] == b[1][both]).all()


def test_multithreaded_port_tcf_no_false_negatives(oracle):
    keys = wl.keys_without_sentinels(21, 50000)
    t = oracle.OracleTable(1, 4, [(1 << 16, 16, 2, 1, 0), ((1 << 16) // 100, 4, 20, 0, 0)], 42)
    ok = t.insert_many(keys, wl.values_for(keys, 2, 1).astype(np.uint64), threads=4)
    f, _ = t.query_many(keys, threads=4)
    assert (f | ~ok).all()


@pytest.mark.parametrize("name", sorted(BCASES))
def test_bucketed_oracle_matches_reference_golden(oracle, name):
    """Every step of the recorded script (insert, query, remove, insert_with_delete,
    insert_if_not_exists, insert_if_not_exists_delete): results and both levels'
    bytes equal the reference's."""
    g = golden(name)
    if g is None:
        pytest.skip(f"golden fixture ref_{name}.npz not recorded yet")
    o = oracle_btable(oracle, name)
    for s in range(int(g["steps"][0])):
        ok, out, fd = o.bulk(int(g[f"s{s}_op"][0]), g[f"s{s}_keys"], g[f"s{s}_vals"])
        assert (ok == g[f"s{s}_ok"].astype(bool)).all(), f"step {s} ok"
        assert (out == g[f"s{s}_out"]).all(), f"step {s} values"
        assert (fd == g[f"s{s}_found"].astype(bool)).all(), f"step {s} found"
        for l in range(2):
            assert o.level_bytes(l) == g[f"s{s}_dump_l{l}"].tobytes(), f"step {s} level {l} bytes"


def test_bucketed_tags_and_tombstone_reuse(oracle):
    """Tags move 0 and all-ones off the sentinels; a removed slot is reused only
    by insert_with_delete; insert_if_not_exists reports the stored value."""
    assert oracle.lib().pgo_btag(16, 0x10000) == 1 and oracle.lib().pgo_btag(16, 0xFFFF) == 0xFFFE
    assert oracle.lib().pgo_btag(8, 0x100) == 1 and oracle.lib().pgo_btag(8, 0x1FF) == 0xFE
    o = oracle.OracleBucketed(16, [(16, 16, 2, 2, 3)], 7)
    keys = wl.keys_without_sentinels(5, 16)
    ok, _, _ = o.bulk(oracle.BOP_INSERT, keys, keys & np.uint64(0xFF))
    assert ok.sum() >= 12 and o.count_fill(0) == ok.sum()
    placed = keys[ok]
    r, _, _ = o.bulk(oracle.BOP_REMOVE, placed[:4])
    assert r.all() and o.count_fill(0) == ok.sum() - 4
    new = wl.keys_without_sentinels(6, 4)
    before = o.level_bytes(0)
    ok2, _, _ = o.bulk(oracle.BOP_INSERT_DELETE, new, np.arange(4, dtype=np.uint64))
    assert ok2.all() and o.level_bytes(0) != before
    f, v, found = o.bulk(oracle.BOP_INSERT_IF_NOT_EXISTS, new[:1], np.array([99], dtype=np.uint64))
    assert f[0] and found[0] and v[0] == 0


@pytest.mark.parametrize("bits", [16, 8])
def test_bucketed_oracle_sawtooth_keeps_its_fill(oracle, bits):
    """The reference's sawtooth flow (tests/src/sawtooth_test.cu:624-826) on the
    oracle: fill to 0.9 of a 2^14-slot filter with 2 % backing, then rounds of
    removing half the live keys, querying the other half and re-adding fresh
    keys with insert_with_delete.  After every round the live fill (both
    levels) equals placed - removed + re-added, every queried key that was
    placed and not removed by a same-tag neighbour is found, and re-adds reuse
    the tombstones (the occupied count does not grow past the fill)."""
    import poggers_b200 as pg
    n0 = 1 << 14
    cfg = pg.data_structs.del_tcf(n0, 2 * n0 // 100, tag_bits=bits)
    levels = [(L.nslots, L.bucket_size, L.max_probes, L.scheme, L.probe) for L in cfg.levels]
    o = oracle.OracleBucketed(bits, levels, 42)
    mask = np.uint64((1 << bits) - 1)
    n = int(0.9 * n0)
    half = n // 2
    live = wl.keys_without_sentinels(91, n)
    vals = wl.values_for(live, 2, 92).astype(np.uint64) & mask
    ok, _, _ = o.bulk(oracle.BOP_INSERT, live, vals)
    placed = int(ok.sum())
    occupied0 = o.count_fill(0) + o.count_fill(1)
    assert occupied0 == placed
    for rnd in range(3):
        r, _, _ = o.bulk(oracle.BOP_REMOVE, live[:half])
        f, _, _ = o.bulk(oracle.BOP_QUERY, live[half:])
        fresh = wl.keys_without_sentinels(1000 + rnd, half)
        fv = wl.values_for(fresh, 2, 2000 + rnd).astype(np.uint64) & mask
        a, _, _ = o.bulk(oracle.BOP_INSERT_DELETE, fresh, fv)
        placed += int(a.sum()) - int(r.sum())
        assert o.count_fill(0) + o.count_fill(1) == placed, f"round {rnd}"
        live[:half], vals[:half] = fresh, fv
        # a query misses only where a remove took a same-tag slot of another key
        assert (~f).sum() <= (20 if bits == 16 else 400), (rnd, int((~f).sum()))


# ---- the reference's slab allocator, restated (oracle/poggers_oracle_slabref.c)
# Known answers derived from the reference's code paths (slab_one_size.cuh:186-288,
# offset_slab.cuh:330-675, 1466-1780).
NULL = (1 << 64) - 1


def _fill_groups(a, sm, ngroups, group=32):
    got, nulls = [], 0
    for _ in range(ngroups):
        o, n = a.malloc(sm, group)
        got += [int(x) for x in o if x != NULL]
        nulls += n
    return got, nulls


def test_refslab_pins_at_creation_and_counts_the_pool(oracle):
    a = oracle.RefSlab(300 * 4096, sms=148, extra_blocks=1)
    assert a.report_max() == 300 and a.report_fill() == 300 - 148 * 2 and a.short_pins == 0
    # the reference's own test flow is over-provisioned: 15M + n + 4096 objects, 16 pins per SM
    b = oracle.RefSlab(15000000 + (1 << 20) + 4096, sms=148, extra_blocks=15)
    assert b.report_fill() == b.report_max() - 148 * 16
    got, nulls = [], 0
    for g in range((1 << 20) // 32):
        o, n = b.malloc(g % 148, 32)
        got += [int(x) for x in o]
        nulls += n
    assert nulls == 0 and len(set(got)) == 1 << 20 and max(got) < b.report_max() * 4096


def test_refslab_without_backups_never_uses_the_pool(oracle):
    # E = 0: one pinned slab; its 4096 objects, then every malloc fails
    # (the pivot finds no backup and leaves the primary place busy)
    a = oracle.RefSlab(2 * 4096, sms=1, extra_blocks=0)
    got, nulls = _fill_groups(a, 0, 128)
    assert nulls == 0 and len(set(got)) == 4096 and all(x // 4096 == got[0] // 4096 for x in got)
    o, n = a.malloc(0, 32)
    assert n == 32 and a.report_fill() == 1
    o, n = a.malloc(0, 1)
    assert n == 1


def test_refslab_pivot_refills_from_the_pool_then_returns_null(oracle):
    # E = 1, three slabs: A (primary) and B (backup) pinned, C in the pool
    a = oracle.RefSlab(3 * 4096, sms=1, extra_blocks=1)
    assert a.report_fill() == 1
    got, nulls = _fill_groups(a, 0, 128)          # A: 4096 objects
    assert nulls == 0 and a.report_fill() == 1
    o, n = a.malloc(0, 32)                          # A has no whole word: B becomes primary, C refills
    assert n == 0 and a.report_fill() == 0
    got += [int(x) for x in o]
    got2, nulls = _fill_groups(a, 0, 127)           # the rest of B
    assert nulls == 0
    o, n = a.malloc(0, 32)                          # B exhausted, C primary, the pool is empty:
    assert n == 1                                   # the pivot's winner returns NULL, the others retry on C
    got2 += [int(x) for x in o if x != NULL]
    more, nulls = _fill_groups(a, 0, 140)           # the rest of C, then NULL: no backup is left
    every = got + got2 + more
    assert len(every) == 3 * 4096 and len(set(every)) == len(every)
    o, n = a.malloc(0, 32)
    assert n == 32


def test_refslab_free_returns_only_empty_unpinned_slabs(oracle):
    a = oracle.RefSlab(3 * 4096, sms=1, extra_blocks=1)
    first, _ = _fill_groups(a, 0, 128)              # slab A full
    a.malloc(0, 32)                                 # A unpinned, B primary, C taken: pool empty
    assert a.report_fill() == 0
    codes = [a.free(x) for x in first]
    assert codes.count(oracle.RSLAB_RETURNED) == 1 and codes[-1] == oracle.RSLAB_RETURNED
    assert codes.count(oracle.RSLAB_REFUSED) == 0 and a.report_fill() == 1
    assert a.free(first[0]) == oracle.RSLAB_REFUSED  # a double free changes nothing
    assert a.report_fill() == 1
    # a pinned slab emptied by frees stays out of the pool; bits of a claimed
    # word still in the SM's cache keep the slab from being empty
    b = oracle.RefSlab(2 * 4096, sms=1, extra_blocks=0)
    got, _ = _fill_groups(b, 0, 3)                  # words 1 and 2 claimed; 32 bits of word 2 cached
    codes = [b.free(x) for x in got]
    assert codes.count(oracle.RSLAB_EMPTIED_PINNED) == 0 and codes.count(oracle.RSLAB_RETURNED) == 0
    c = oracle.RefSlab(2 * 4096, sms=1, extra_blocks=0)
    got, _ = _fill_groups(c, 0, 4)                  # the cache drained: both words handed out
    codes = [c.free(x) for x in got]
    assert codes.count(oracle.RSLAB_EMPTIED_PINNED) == 1 and codes[-1] == oracle.RSLAB_EMPTIED_PINNED
    assert c.report_fill() == 1
