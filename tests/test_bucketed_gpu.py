"""GPU parity tests of the bucketed filter with tombstone reuse (packed slots).

Bar: in the serial launch shape every step of the script recorded from the
reference's CUDA build (insert, query, remove, insert_with_delete,
insert_if_not_exists, insert_if_not_exists_delete) gives the reference's
results and the reference's bytes in both levels.  In the parallel shape the
reference's delete-test flow gives no false negatives, no failed removes or
re-adds, and tag-collision counts within a stated tolerance of the
reference's own parallel run.
"""
import json

import numpy as np
import pytest

from tests.cases import BCASES, GOLDEN, golden
from tests.gpu_util import to_dev
from poggers_b200 import workload as wl

pytestmark = pytest.mark.gpu

OPS = ("insert", "query", "remove", "insert_delete", "insert_if_not_exists", "insert_if_not_exists_delete")


def _table(pg, name):
    bits, levels, seed = BCASES[name]
    fmt = pg.FMT_PACKED_TAGVAL16 if bits == 16 else pg.FMT_PACKED_TAGVAL8
    cfg = pg.TableConfig(fmt, 4, [pg.Level(*lv) for lv in levels])
    return pg.Table(cfg, seed), bits


def _vals_dev(bits, v):
    import torch
    if bits == 16:
        return torch.from_numpy(np.ascontiguousarray(v).astype(np.uint16).view(np.int16)).cuda()
    return torch.from_numpy(np.ascontiguousarray(v).astype(np.uint8)).cuda()


def _run(pg, t, bits, op, keys, vals=None):
    """One bulk operation; returns (ok, out values, found) as numpy."""
    import torch
    n = len(keys)
    k = to_dev(np.ascontiguousarray(keys, dtype=np.uint64))
    v = None if vals is None else _vals_dev(bits, vals)
    ok = torch.zeros(n, dtype=torch.uint8, device="cuda")
    out = torch.zeros(n, dtype=torch.int16 if bits == 16 else torch.uint8, device="cuda")
    fd = torch.zeros(n, dtype=torch.uint8, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    if op == 0:
        t.bulk_insert(k, v, ok, cnt)
    elif op == 1:
        t.bulk_query(k, out, ok, cnt)
    elif op == 2:
        t.bulk_remove(k, ok, cnt)
    elif op == 3:
        t.bulk_insert_with_delete(k, v, ok, cnt)
    else:
        t.bulk_insert_if_not_exists(k, v, out, fd, ok, cnt, delete=(op == 5))
    torch.cuda.synchronize()
    okn = ok.cpu().numpy().astype(bool)
    c = int(cnt.item())
    assert c == (int(okn.sum()) if op in (1, 2) else int((~okn).sum())), "counter disagrees with the flags"
    o = out.cpu().numpy()
    o = (o.view(np.uint16) if bits == 16 else o).astype(np.uint64)
    return okn, o, fd.cpu().numpy().astype(bool)


@pytest.mark.parametrize("lanes", [1, 4])
@pytest.mark.parametrize("name", sorted(BCASES))
def test_serial_matches_reference_script_bytes(pg, name, lanes):
    g = golden(name)
    if g is None:
        pytest.skip(f"golden fixture ref_{name}.npz not recorded yet")
    t, bits = _table(pg, name)
    t.serial(lanes)
    for s in range(int(g["steps"][0])):
        op = int(g[f"s{s}_op"][0])
        vals = g[f"s{s}_vals"] if op in (0, 3, 4, 5) else None
        ok, out, fd = _run(pg, t, bits, op, g[f"s{s}_keys"], vals)
        assert (ok == g[f"s{s}_ok"].astype(bool)).all(), f"step {s} ({OPS[op]}) ok"
        if op in (1, 4, 5):
            assert (out == g[f"s{s}_out"]).all(), f"step {s} ({OPS[op]}) values"
        if op in (4, 5):
            assert (fd == g[f"s{s}_found"].astype(bool)).all(), f"step {s} ({OPS[op]}) found"
        for lv in range(2):
            assert t.dump_level(lv) == g[f"s{s}_dump_l{lv}"].tobytes(), f"step {s} ({OPS[op]}) level {lv} bytes"


@pytest.mark.parametrize("name", sorted(BCASES))
def test_parallel_matches_oracle_on_a_script(pg, oracle, name):
    """Phase-separated parallel launches against the sequential oracle: every key
    placed by both runs answers queries alike; removes and re-adds succeed for the
    same keys; fill counts agree up to the keys whose placement differs."""
    bits, levels, seed = BCASES[name]
    t, _ = _table(pg, name)
    o = oracle.OracleBucketed(bits, levels, seed)
    n = 3000
    keys = wl.keys_without_sentinels(77, n)
    vals = wl.values_for(keys, 2, 3).astype(np.uint64) & np.uint64((1 << bits) - 1)
    ok, _, _ = _run(pg, t, bits, 0, keys, vals)
    oko, _, _ = o.bulk(oracle.BOP_INSERT, keys, vals)
    assert ok.all() and oko.all()
    f, v, _ = _run(pg, t, bits, 1, keys)
    assert f.all(), "false negatives"
    # a remove takes the first slot holding the key's tag, which with short
    # tags is sometimes another key's: both runs remove (almost) every key
    r, _, _ = _run(pg, t, bits, 2, keys[: n // 2])
    ro, _, _ = o.bulk(oracle.BOP_REMOVE, keys[: n // 2])
    assert abs(int(r.sum()) - int(ro.sum())) <= 5 and r.mean() > 0.99
    occ, tomb = t.get_fill(0)
    occ1, tomb1 = t.get_fill(1)
    assert (occ - tomb) + (occ1 - tomb1) == n - int(r.sum())
    assert o.count_fill(0) + o.count_fill(1) == n - int(ro.sum())
    a, _, _ = _run(pg, t, bits, 3, keys[: n // 2], vals[: n // 2])
    assert a.all()
    occ, tomb = t.get_fill(0)
    occ1, tomb1 = t.get_fill(1)
    assert (occ - tomb) + (occ1 - tomb1) == n - int(r.sum()) + n // 2


def _ref_stats():
    p = GOLDEN / "ref_bucketed_stats.json"
    return json.loads(p.read_text()) if p.exists() else None


@pytest.mark.parametrize("name,bits", [("del_tcf", 16), ("del_tcf_small", 8)])
def test_delete_flow_matches_reference_statistics(pg, name, bits):
    """The reference's delete test (tests/src/delete_tests.cu:568-760) at 2^22
    primary slots + 1% backing, 0.9 load, parallel launches.  Zero insert
    failures, as the reference's run.  A remove takes the first slot holding
    the key's tag, sometimes another key's, so failed removes, false negatives
    and failed re-adds may occur in either library: each within 10 of the
    reference's count; tag-collision value mismatches within 25% (+20) of the
    reference's (which key a shared tag answers for depends on the order)."""
    stats = _ref_stats()
    n0 = 1 << 22
    n1 = n0 // 100
    n = int(0.9 * (n0 + n1))
    mask = (1 << bits) - 1
    keys = wl.keys_without_sentinels(42, n)
    vals = wl.values_for(keys, 2, 49).astype(np.uint64) & np.uint64(mask)
    t = pg.Table(pg.data_structs.del_tcf(n0, n1, tag_bits=bits), 42)
    half = n // 2
    ok, _, _ = _run(pg, t, bits, 0, keys, vals)
    r, _, _ = _run(pg, t, bits, 2, keys[:half])
    qf, qv, _ = _run(pg, t, bits, 1, keys[half:])
    a, _, _ = _run(pg, t, bits, 3, keys[:half], vals[:half])
    af, _, _ = _run(pg, t, bits, 1, keys)
    mism = int((qf & (qv != vals[half:])).sum())
    fn = int((~qf & ok[half:]).sum())
    assert (~ok).sum() == 0
    assert (~r).sum() <= 10 and fn <= 10 and (~a).sum() <= 10 and (~af).sum() <= 20
    if stats is not None:
        ref = stats[name]
        assert ref["insert_failures"] == 0
        assert abs(int((~r).sum()) - ref["remove_misses"]) <= 10
        assert abs(fn - ref["query_misses"]) <= 10
        assert abs(int((~a).sum()) - ref["readd_failures"]) <= 10
        assert abs(mism - ref["query_value_mismatches"]) <= 0.25 * ref["query_value_mismatches"] + 20


def test_insert_if_not_exists_reports_present_keys(pg):
    import torch
    t = pg.Table(pg.data_structs.del_tcf(1 << 16, 1 << 10), 5)
    keys = wl.keys_without_sentinels(8, 40000)
    vals = wl.values_for(keys, 2, 4).astype(np.uint64) & np.uint64(0xFFFF)
    ok, _, _ = _run(pg, t, 16, 0, keys[:20000], vals[:20000])
    assert ok.all()
    ok2, out, fd = _run(pg, t, 16, 4, keys, (vals + 1) & np.uint64(0xFFFF))
    assert ok2.all() and fd[:20000].all()
    # a present key reports a stored value of its tag (its own unless a tag collides)
    assert (out[:20000] == vals[:20000]).mean() > 0.99
    # absent keys were inserted unless a colliding tag already answered for them
    assert fd[20000:].mean() < 0.05
    f, _, _ = _run(pg, t, 16, 1, keys)
    assert f.all()
    # the _delete form removes what it finds
    ok3, _, fd3 = _run(pg, t, 16, 5, keys[:1000], vals[:1000])
    assert ok3.all() and fd3.all()
    occ, tomb = t.get_fill(0)
    assert tomb >= 900
    del torch


def test_packed_formats_reject_unsupported_calls(pg):
    import torch
    t = pg.Table(pg.data_structs.hash_table_64(1 << 12, bucket=8), 1)
    k = to_dev(wl.keys_without_sentinels(1, 10))
    with pytest.raises(pg.PoggersError):
        t.bulk_insert_with_delete(k)
    # one batch serves tables of one kernel shape: a filter and a hash table do not mix
    with pytest.raises(pg.PoggersError):
        pg.Batch([pg.Table(pg.data_structs.del_tcf(1 << 12, 64), 1), t], 16)
    del torch


def _sawtooth(run, bits, n, half, mask, rounds=3):
    """One sawtooth run through run(op, keys, vals) -> (ok, out, found): the fill,
    then rounds of remove / query / insert_with_delete.  Returns the per-phase
    results and the live keys' history."""
    live = wl.keys_without_sentinels(91, n)
    vals = wl.values_for(live, 2, 92).astype(np.uint64) & mask
    steps = [("insert", run(0, live, vals))]
    for rnd in range(rounds):
        steps.append(("remove", run(2, live[:half], None)))
        steps.append(("query", run(1, live[half:], None)))
        fresh = wl.keys_without_sentinels(1000 + rnd, half)
        fv = wl.values_for(fresh, 2, 2000 + rnd).astype(np.uint64) & mask
        steps.append(("insert_delete", run(3, fresh, fv)))
        live[:half], vals[:half] = fresh, fv
    return steps


def _counts(steps):
    c = {"insert_fail": 0, "remove_miss": 0, "false_neg": 0, "readd_fail": 0}
    for name, (ok, _, _) in steps:
        key = {"insert": "insert_fail", "remove": "remove_miss", "query": "false_neg",
               "insert_delete": "readd_fail"}[name]
        c[key] += int((~ok).sum())
    return c


@pytest.mark.parametrize("bits", [16, 8])
def test_sawtooth_rounds(pg, oracle, bits):
    """The reference's sawtooth test (tests/src/sawtooth_test.cu:624-826, whose
    main runs the 8-bit filter with 2 % backing, 50 % per round): fill the
    bucketed filter to 0.9, then rounds of removing the first half of the live
    keys, querying the other half, and re-adding fresh keys in their place with
    insert_with_delete.  The serial launch gives the sequential oracle's
    results (every flag and value) and bytes in both levels after every round.
    The parallel launch's counts (insert and re-add failures, removes that found
    nothing, false negatives) are compared with the reference's own parallel
    build on the same keys: a table this small has every key of a batch in
    flight at once, so both differ from the sequential order."""
    import torch
    from oracle import pyrefcuda as rc
    n0 = 1 << 14
    n1 = 2 * n0 // 100
    cfg = pg.data_structs.del_tcf(n0, n1, tag_bits=bits)
    levels = [(L.nslots, L.bucket_size, L.max_probes, L.scheme, L.probe) for L in cfg.levels]
    mask = np.uint64((1 << bits) - 1)
    n = int(0.9 * n0)
    half = n // 2
    # serial: the oracle's results and bytes after every step
    t = pg.Table(cfg, 42)
    t.serial(1)
    o = oracle.OracleBucketed(bits, levels, 42)
    dumps = []

    def run_serial(op, k, v):
        r = _run(pg, t, bits, op, k, v)
        dumps.append((t.dump_level(0), t.dump_level(1)))
        return r

    mine = _sawtooth(run_serial, bits, n, half, mask)
    odumps = []

    def run_oracle(op, k, v):
        r = o.bulk(op, k, v)
        odumps.append((o.level_bytes(0), o.level_bytes(1)))
        return r

    ref = _sawtooth(run_oracle, bits, n, half, mask)
    for s, ((name, (ok, out, _)), (_, (oko, oout, _))) in enumerate(zip(mine, ref)):
        assert (ok == oko).all(), f"step {s} ({name}) flags"
        if name == "query":
            assert (out[ok] == oout[ok]).all(), f"step {s} values"
        assert dumps[s] == odumps[s], f"step {s} ({name}) bytes"
    t.free_on_device()
    # parallel: counts against the reference's own parallel build
    t = pg.Table(cfg, 42)
    par = _counts(_sawtooth(lambda op, k, v: _run(pg, t, bits, op, k, v), bits, n, half, mask))
    t.free_on_device()
    torch.cuda.synchronize()
    if not rc.available():
        pytest.skip("the reference's CUDA build is not built here; serial parity checked")
    kind = rc.KIND_DEL_TCF if bits == 16 else rc.KIND_DEL_TCF_SMALL
    r = rc.RefTable(kind, n0, n1, 42)

    def run_ref(op, k, v):
        import torch as th
        dk = to_dev(np.ascontiguousarray(k, dtype=np.uint64))
        dv = None if v is None else _vals_dev(bits, v)
        ok = th.zeros(len(k), dtype=th.uint8, device="cuda")
        out = th.zeros(len(k), dtype=th.int16 if bits == 16 else th.uint8, device="cuda")
        r.bbulk(op if op != 3 else rc.OP_INSERT_DELETE, dk, dv, ok, out)
        th.cuda.synchronize()
        return ok.cpu().numpy().astype(bool), None, None

    refc = _counts(_sawtooth(run_ref, bits, n, half, mask))
    r.close()
    print("parallel counts, ours", par, "reference build", refc)
    for k in par:
        assert par[k] <= 1.5 * refc[k] + 32, (k, par, refc)
