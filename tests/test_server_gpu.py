"""GPU tests of the continuous-batching server.

Requests are submitted while earlier ones are still on the GPU; each result
must equal what the same request returns when the requests run one at a time
in submission order through the plain per-request path (pg_bulk_* on identical
tables).  uint64 tables: bit-exact (loads stay below the point where inserts
fail).  Filters: every inserted key found in both runs, with its own value
except where another key's equal 16-bit tag sits earlier in its buckets
(placement, hence such collisions and false positives, depends on the order
of concurrent inserts in either path)."""
import numpy as np
import pytest

from tests.gpu_util import Driver
from poggers_b200 import workload as wl

pytestmark = pytest.mark.gpu


def _stream(rng, ntables, nreq, sizes, kinds):
    """Seeded request stream: (table, op, keys) with Zipf-ish table choice."""
    inserted = [[] for _ in range(ntables)]
    fresh = [0] * ntables
    reqs = []
    w = 1.0 / np.arange(1, ntables + 1) ** 0.99
    w /= w.sum()
    for _ in range(nreq):
        t = int(rng.choice(ntables, p=w))
        n = int(np.exp(rng.uniform(0, np.log(3000))))
        cap = int(0.6 * sizes[t]) - sum(len(x) for x in inserted[t])
        u = rng.uniform()
        if u < 0.3 and cap > n:
            k = wl.keys_without_sentinels(10_000 * t + 17, fresh[t] + n)[fresh[t]:]
            fresh[t] += n
            inserted[t].append(k)
            reqs.append((t, 0, k))
        elif u < 0.9 or kinds[t] == "tcf":
            have = np.concatenate(inserted[t]) if inserted[t] else np.zeros(0, dtype=np.uint64)
            pos = have[rng.integers(0, len(have), n // 2)] if len(have) else np.zeros(0, dtype=np.uint64)
            neg = wl.keys_without_sentinels(7_000_000 + rng.integers(1 << 30), n - len(pos))
            reqs.append((t, 1, np.concatenate([pos, neg])))
        else:
            have = np.concatenate(inserted[t]) if inserted[t] else np.zeros(0, dtype=np.uint64)
            if len(have) == 0:
                continue
            reqs.append((t, 2, have[rng.integers(0, len(have), max(1, n // 4))]))
    return reqs


def test_server_results_equal_sequential_plain_path(pg):
    import torch
    rng = np.random.default_rng(11)
    kinds = ["ht"] * 6 + ["ht_fp"] * 3 + ["tcf"] * 5
    sizes = [int(2 ** rng.uniform(13, 17)) for _ in kinds]

    def cfg(kind, n):
        if kind == "tcf":
            return pg.data_structs.tcf(n, max(n // 100, 16))
        c = pg.data_structs.hash_table_64(n, bucket=8)
        c.fingerprints = kind == "ht_fp"
        return c

    srv = pg.Server(hbm_budget_bytes=1 << 34, max_wave_keys=1 << 16, max_wave_requests=256)
    ids = [srv.add_table(cfg(k, n), 50 + i) for i, (k, n) in enumerate(zip(kinds, sizes))]
    plain = [pg.Table(cfg(k, n), 50 + i) for i, (k, n) in enumerate(zip(kinds, sizes))]
    reqs = _stream(rng, len(kinds), 400, sizes, kinds)
    outs = []
    rids = []
    for t, op, keys in reqs:
        vb = 8 if kinds[t] != "tcf" else 2
        vals = wl.values_for(keys, vb, 3) if op == 0 else None
        vout = np.zeros(len(keys), dtype=np.uint64 if vb == 8 else np.uint16)
        flags = np.zeros(len(keys), dtype=np.uint8)
        rids.append(srv.submit(ids[t], op, keys, vals, vout, flags))
        outs.append((vals, vout, flags))
    res = [srv.poll(r, wait=True) for r in rids]
    waves, nkeys = srv.stats()
    assert waves < len(reqs), "requests should share waves"
    assert nkeys == sum(len(k) for _, _, k in reqs)
    inserted = [set() for _ in kinds]
    value_of = [dict() for _ in kinds]
    tcf_known = tcf_own_served = tcf_own_plain = 0
    for (t, op, keys), (vals, vout, flags), (count, lat) in zip(reqs, outs, res):
        d = Driver(plain[t])
        f = flags.astype(bool)
        assert lat >= 0
        if op == 0:
            ok = d.insert(keys, vals.astype(np.uint64))
            if kinds[t] != "tcf":
                assert (f == ok).all() and f.all()
            assert count == (~f).sum()
            inserted[t].update(map(int, keys[f]))
            for k, v in zip(keys[f], vals[f]):
                value_of[t][int(k)] = int(v)
        elif op == 1:
            fo, vo = d.query(keys)
            if kinds[t] == "tcf":
                # every key inserted and not removed is found by both paths;
                # its value is its own unless another key with the same 16-bit
                # tag sits earlier in its buckets (the reference returns the
                # first match, and placement differs between the two paths)
                known = np.array([int(k) in inserted[t] for k in keys], dtype=bool)
                assert f[known].all() and fo[known].all()
                own = np.array([value_of[t].get(int(k), -1) for k in keys[known]], dtype=np.int64)
                tcf_known += int(known.sum())
                tcf_own_served += int((vout[known].astype(np.int64) == own).sum())
                tcf_own_plain += int((vo[known].astype(np.int64) == own).sum())
            else:
                assert (f == fo).all() and (vout.astype(np.uint64) == vo).all()
            assert count == f.sum()
        else:
            ro = d.remove(keys)
            # a request may name a key twice: one of the two removes it, and which
            # one depends on the order inside the launch, in either path
            u, inv = np.unique(keys, return_inverse=True)
            got_s = np.zeros(len(u), dtype=int)
            got_p = np.zeros(len(u), dtype=int)
            np.add.at(got_s, inv, f.astype(int))
            np.add.at(got_p, inv, ro.astype(int))
            assert (got_s == got_p).all() and got_s.max(initial=0) <= 1
            assert count == f.sum()
            for k in keys[f]:
                inserted[t].discard(int(k))
    # tag collisions are ~0.04 % per key at these loads
    assert tcf_known > 1000
    assert tcf_own_served >= 0.999 * tcf_known and tcf_own_plain >= 0.999 * tcf_known
    srv.close()


def test_server_admits_tables_by_hbm_budget(pg):
    srv = pg.Server(hbm_budget_bytes=64 << 20, max_wave_keys=1 << 12, max_wave_requests=16)
    cfg = pg.data_structs.hash_table_64(1 << 20, bucket=8)   # 16 MiB
    got = [srv.add_table(cfg, i) for i in range(6)]
    assert got[:4] == [0, 1, 2, 3] and got[4] is None and got[5] is None
    assert srv.bytes_in_use() == 4 * (16 << 20)
    srv.drop_table(1)
    assert srv.add_table(cfg, 9) is not None
    t = srv.add_table(pg.data_structs.hash_table_64(1 << 10, bucket=8), 3)
    assert t is None
    k = wl.keys_without_sentinels(5, 100)
    f = np.zeros(100, dtype=np.uint8)
    r = srv.submit(0, 0, k, wl.values_for(k, 8, 1), None, f)
    assert srv.poll(r, wait=True)[0] == 0 and f.all()
    # a collected id, or one never issued, is refused instead of waited on
    for bad in (r, r + 1000):
        with pytest.raises(pg.PoggersError):
            srv.poll(bad, wait=True)
    srv.close()


def test_server_serves_bucketed_filters(pg):
    """A 16-bit bucketed filter behind the serving loop: inserts, queries,
    removes and insert_with_delete requests, each result as the table's own
    bulk call would give it."""
    srv = pg.Server(hbm_budget_bytes=1 << 30, max_wave_keys=1 << 16, max_wave_requests=64)
    try:
        tid = srv.add_table(pg.data_structs.del_tcf(1 << 16, 1 << 10), 7)
        assert tid is not None
        keys = wl.keys_without_sentinels(21, 40000)
        vals = (wl.values_for(keys, 2, 22).astype(np.uint64) & np.uint64(0xFFFF)).astype(np.uint16)
        fl = np.zeros(len(keys), dtype=np.uint8)
        srv.poll(srv.submit(tid, pg.PG_OP_INSERT, keys, vals, None, fl), wait=True)
        assert fl.all()
        vo = np.zeros(len(keys), dtype=np.uint16)
        fq = np.zeros(len(keys), dtype=np.uint8)
        srv.poll(srv.submit(tid, pg.PG_OP_QUERY, keys, None, vo, fq), wait=True)
        assert fq.all() and (vo == vals).mean() > 0.999
        fr = np.zeros(20000, dtype=np.uint8)
        srv.poll(srv.submit(tid, pg.PG_OP_REMOVE, keys[:20000], None, None, fr), wait=True)
        assert fr.all()
        fa = np.zeros(20000, dtype=np.uint8)
        srv.poll(srv.submit(tid, pg.PG_OP_INSERT_WITH_DELETE, keys[:20000], vals[:20000], None, fa), wait=True)
        assert fa.all()
        fq2 = np.zeros(len(keys), dtype=np.uint8)
        srv.poll(srv.submit(tid, pg.PG_OP_QUERY, keys, None, None, fq2), wait=True)
        assert fq2.all()
    finally:
        srv.close()


def test_server_serves_8bit_filters_beside_16bit_ones(pg):
    """An 8-bit and a 16-bit bucketed filter served in the same waves (their
    values staged at their own widths), against twin tables driven by the bulk
    calls: every insert and re-add placed, no false negatives, and the 8-bit
    filter's values agree with its twin's as often as tag collisions allow."""
    import torch
    from tests.gpu_util import to_dev
    srv = pg.Server(hbm_budget_bytes=1 << 30, max_wave_keys=1 << 16, max_wave_requests=64)
    try:
        c8 = pg.data_structs.del_tcf(1 << 15, 1 << 9, tag_bits=8)
        c16 = pg.data_structs.del_tcf(1 << 15, 1 << 9)
        t8, t16 = srv.add_table(c8, 8), srv.add_table(c16, 16)
        assert t8 is not None and t16 is not None
        keys = wl.keys_without_sentinels(31, 24000)
        v8 = (wl.values_for(keys, 2, 32).astype(np.uint64) & np.uint64(0xFF)).astype(np.uint8)
        v16 = (wl.values_for(keys, 2, 33).astype(np.uint64) & np.uint64(0xFFFF)).astype(np.uint16)
        f8, f16 = np.zeros(len(keys), np.uint8), np.zeros(len(keys), np.uint8)
        # submitted back to back, so both requests can join one wave
        r8 = srv.submit(t8, pg.PG_OP_INSERT, keys, v8, None, f8)
        r16 = srv.submit(t16, pg.PG_OP_INSERT, keys, v16, None, f16)
        srv.poll(r8, wait=True), srv.poll(r16, wait=True)
        assert f8.all() and f16.all()
        q8, q16 = np.zeros(len(keys), np.uint8), np.zeros(len(keys), np.uint16)
        g8, g16 = np.zeros(len(keys), np.uint8), np.zeros(len(keys), np.uint8)
        r8 = srv.submit(t8, pg.PG_OP_QUERY, keys, None, q8, g8)
        r16 = srv.submit(t16, pg.PG_OP_QUERY, keys, None, q16, g16)
        srv.poll(r8, wait=True), srv.poll(r16, wait=True)
        assert g8.all() and g16.all()
        assert (q16 == v16).mean() > 0.999
        fr = np.zeros(12000, np.uint8)
        srv.poll(srv.submit(t8, pg.PG_OP_REMOVE, keys[:12000], None, None, fr), wait=True)
        # a remove takes the first slot with the key's tag, sometimes another key's:
        # with 8-bit tags a few removes can find none left
        assert fr.sum() >= 12000 - 10
        fa = np.zeros(12000, np.uint8)
        srv.poll(srv.submit(t8, pg.PG_OP_INSERT_WITH_DELETE, keys[:12000], v8[:12000], None, fa), wait=True)
        assert fa.all()

        # the twin: the same filter through the bulk calls
        tw = pg.Table(c8, 8)
        dk = to_dev(keys)
        ok = torch.zeros(len(keys), dtype=torch.uint8, device="cuda")
        tw.bulk_insert(dk, torch.from_numpy(v8).cuda(), ok)
        tv = torch.zeros(len(keys), dtype=torch.uint8, device="cuda")
        tf = torch.zeros(len(keys), dtype=torch.uint8, device="cuda")
        tw.bulk_query(dk, tv, tf)
        torch.cuda.synchronize()
        assert ok.all() and tf.all()
        twin_match = (tv.cpu().numpy() == v8).mean()
        assert abs((q8 == v8).mean() - twin_match) < 0.01, ((q8 == v8).mean(), twin_match)
        tw.free_on_device()
    finally:
        srv.close()


def test_server_large_requests_split_their_host_copies(pg):
    """Requests of 2^21 keys (16 MiB of keys and as much of values, so the
    wave's host copies are split over several threads) on a uint64 table with
    fingerprints: every insert placed, every query answered with its value,
    absent keys not found, removes seen by the next query; the table dropped
    afterwards."""
    srv = pg.Server(hbm_budget_bytes=4 << 30, max_wave_keys=1 << 22, max_wave_requests=64)
    try:
        cfg = pg.data_structs.hash_table_64(1 << 23, bucket=8)
        cfg.fingerprints = True
        tid = srv.add_table(cfg, 9)
        n = 1 << 21
        keys = wl.keys_without_sentinels(81, n)
        vals = wl.values_for(keys, 8, 82)
        fl = np.zeros(n, dtype=np.uint8)
        srv.poll(srv.submit(tid, pg.PG_OP_INSERT, keys, vals, None, fl), wait=True)
        assert fl.all()
        q = np.concatenate([keys[: n // 2], wl.keys_without_sentinels(83, n // 2)])
        vo = np.zeros(n, dtype=np.uint64)
        fq = np.zeros(n, dtype=np.uint8)
        srv.poll(srv.submit(tid, pg.PG_OP_QUERY, q, None, vo, fq), wait=True)
        assert fq[: n // 2].all() and not fq[n // 2:].any()
        assert (vo[: n // 2] == vals[: n // 2]).all() and (vo[n // 2:] == 0).all()
        fr = np.zeros(n // 4, dtype=np.uint8)
        srv.poll(srv.submit(tid, pg.PG_OP_REMOVE, keys[: n // 4], None, None, fr), wait=True)
        assert fr.all()
        fq2 = np.zeros(n // 2, dtype=np.uint8)
        srv.poll(srv.submit(tid, pg.PG_OP_QUERY, keys[: n // 2], None, None, fq2), wait=True)
        assert not fq2[: n // 4].any() and fq2[n // 4:].all()
        # the worker's time by stage covers the four requests' waves
        tm = srv.timing()
        waves, keys_run = srv.stats()
        assert tm["waves"] == waves >= 4 and tm["requests"] == 4 and tm["keys"] == keys_run == 2 * n + n // 4 + n // 2
        assert all(tm[k] >= 0 for k in tm if k.endswith("_s")) and tm["copy_in_s"] > 0 and tm["copy_out_s"] > 0
        srv.drop_table(tid)
    finally:
        srv.close()


def test_served_slab_requests_beside_table_requests(pg):
    """Slab size-class sets served by the loop: malloc requests return distinct
    objects of the smallest class that fits, free requests refuse nothing, and
    table requests in the same waves keep their results."""
    import numpy as np
    classes = [16, 64, 256, 1024]
    srv = pg.Server(hbm_budget_bytes=4 << 30, max_wave_keys=1 << 16, max_wave_requests=256)
    sid = srv.add_slab_set(classes, [1 << 16] * 4)
    tid = srv.add_table(pg.data_structs.hash_table_64(1 << 14, bucket=8), 5)
    rng = np.random.default_rng(9)
    sizes = [rng.integers(1, 1025, int(n)).astype(np.uint32) for n in rng.integers(1, 4000, 12)]
    outs = [np.zeros(len(z), dtype=np.uint64) for z in sizes]
    keys = wl.keys_without_sentinels(61, 5000)
    vals = wl.values_for(keys, 8, 2)
    rids = []
    for i, (z, o) in enumerate(zip(sizes, outs)):
        rids.append(srv.submit_slab(sid, pg.PG_OP_MALLOC, z, o))
        if i == 3:
            rids.append(srv.submit(tid, pg.PG_OP_INSERT, keys, vals))
    counts = [srv.poll(r, wait=True)[0] for r in rids]
    assert sum(counts) == 0
    allp = np.concatenate(outs)
    assert (allp != 0).all() and len(np.unique(allp)) == len(allp)
    # each object came from the smallest class that fits its size: objects of
    # one class are that class's size apart from each other
    zs = np.concatenate(sizes)
    cls = np.searchsorted(np.array(classes), zs)
    for c, b in enumerate(classes):
        p = np.sort(allp[cls == c])
        if len(p) > 1:
            assert (np.diff(p) % b == 0).all()
    # query the table between frees
    vout = np.zeros(len(keys), dtype=np.uint64)
    frees = [srv.submit_slab(sid, pg.PG_OP_FREE, o) for o in outs[:6]]
    q = srv.submit(tid, pg.PG_OP_QUERY, keys, None, vout)
    frees += [srv.submit_slab(sid, pg.PG_OP_FREE, o) for o in outs[6:]]
    assert all(srv.poll(r, wait=True)[0] == 0 for r in frees)
    hits = srv.poll(q, wait=True)[0]
    assert hits == len(keys) and (vout == vals).all()
    # a second free of the same objects is refused, every one
    again = srv.submit_slab(sid, pg.PG_OP_FREE, outs[0])
    assert srv.poll(again, wait=True)[0] == len(outs[0])
    srv.close()
