"""Record golden vectors from the REFERENCE's own CUDA build.

Run on a machine with a GPU and the prebuilt oracle/_ref/libpoggers_refcuda.so
(built here by `make -C oracle refcuda` from the reference checkout):

    python tests/golden/make_golden.py --out tests/golden

For each case it drives one of the reference's template tables (one tile,
keys in batch order, exactly like the reference's single-tile drivers) and
records: the keys and values, insert results, the raw slot arrays of every
level after the inserts (the reference's device bytes), query results for
inserted and never-inserted keys, remove results, the slot arrays after the
removes, and the queries again.  The serial order makes every byte
deterministic, so the oracle and the product's serial launch shape must
reproduce the dumps exactly.

It also records full-size statistics from the reference's parallel bulk
kernels (one tile per key, 1024-thread blocks): the filter's false-negative
and false-positive counts on the 2^22-slot workload, and order-independent
checksums of the hash table's query results on the 2^26-slot workload.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import pyrefcuda as rc  # noqa: E402
from poggers_b200 import workload as wl  # noqa: E402

SLOT = {rc.KIND_HT_DOUBLE_B8: 16, rc.KIND_HT_ALIAS: 16, rc.KIND_HT_LINEAR_B8: 16, rc.KIND_HT_P2_B8: 16,
        rc.KIND_TCF: 4, rc.KIND_TCQF: 2}
BUCKET = {rc.KIND_HT_DOUBLE_B8: 8, rc.KIND_HT_ALIAS: 16, rc.KIND_HT_LINEAR_B8: 8, rc.KIND_HT_P2_B8: 8,
          rc.KIND_TCF: 16, rc.KIND_TCQF: 16}
U64MAX = (1 << 64) - 1

# name, kind, primary slots, backing slots, seed, #keys, key seed
CASES = [
    ("ht_double_b8", rc.KIND_HT_DOUBLE_B8, 1000, 0, 43, 1000, 1001),
    ("ht_alias_b16", rc.KIND_HT_ALIAS, 2048, 0, 42, 1900, 1002),
    ("ht_linear_b8", rc.KIND_HT_LINEAR_B8, 1000, 0, 44, 1000, 1003),
    ("ht_p2_b8", rc.KIND_HT_P2_B8, 1000, 0, 45, 900, 1004),
    ("tcf", rc.KIND_TCF, 2048, 2048 // 100, 42, 2000, 1005),
    ("tcqf", rc.KIND_TCQF, 2048, 0, 42, 1900, 1006),
]


def edge_keys(keys: np.ndarray, is_filter: bool) -> np.ndarray:
    """Sentinels, duplicates and (for filters) keys whose low 16 bits are 0 or 0xFFFF."""
    e = [0, U64MAX, int(keys[5]), int(keys[6])]
    if is_filter:
        e += [0x1234_0000_0000_0000, 0xABCD_0000_0000_FFFF, (int(keys[7]) & ~0xFFFF) | 0x0001]
    return np.array(e, dtype=np.uint64)


def levels(kind: int, n0: int, n1: int) -> list[int]:
    nb0 = (n0 - 1) // BUCKET[kind] + 1
    out = [nb0 * BUCKET[kind] * SLOT[kind]]
    if kind == rc.KIND_TCF:
        nb1 = (n1 - 1) // 4 + 1
        out.append(nb1 * 4 * SLOT[kind])
    return out


def run_case(torch, name, kind, n0, n1, seed, nkeys, kseed):
    dev = torch.device("cuda")
    is_filter = kind in (rc.KIND_TCF, rc.KIND_TCQF)
    base = wl.keys_without_sentinels(kseed, nkeys)
    keys = np.concatenate([base, edge_keys(base, is_filter)])
    vbytes = 2 if is_filter else 8
    vals = wl.values_for(keys, vbytes, seed=kseed + 7)
    fresh = wl.keys_without_sentinels(kseed + 500, max(200, nkeys // 2))
    qkeys = np.concatenate([keys, fresh])
    rkeys = np.concatenate([keys[: nkeys // 3], fresh[:20], np.array([0], dtype=np.uint64)])

    t = rc.RefTable(kind, n0, n1, seed)
    vt = torch.int16 if vbytes == 2 else torch.int64
    d_keys = torch.from_numpy(keys.view(np.int64)).to(dev)
    d_vals = torch.from_numpy(vals.view(np.int16 if vbytes == 2 else np.int64)).to(dev)
    ok = torch.zeros(len(keys), dtype=torch.uint8, device=dev)
    t.bulk(rc.OP_INSERT, d_keys, d_vals, ok, serial=True)
    torch.cuda.synchronize()
    sizes = levels(kind, n0, n1)
    dump_ins = [np.frombuffer(t.dump(l, b), dtype=np.uint8) for l, b in enumerate(sizes)]

    def query(qk):
        d_q = torch.from_numpy(qk.view(np.int64)).to(dev)
        f = torch.zeros(len(qk), dtype=torch.uint8, device=dev)
        v = torch.zeros(len(qk), dtype=vt, device=dev)
        t.bulk(rc.OP_QUERY, d_q, None, f, v, serial=True)
        torch.cuda.synchronize()
        vv = v.cpu().numpy()
        vv = vv.view(np.uint16) if vbytes == 2 else vv.view(np.uint64)
        return f.cpu().numpy(), vv.astype(np.uint64)

    q_found, q_vals = query(qkeys)
    d_r = torch.from_numpy(rkeys.view(np.int64)).to(dev)
    rok = torch.zeros(len(rkeys), dtype=torch.uint8, device=dev)
    t.bulk(rc.OP_REMOVE, d_r, None, rok, serial=True)
    torch.cuda.synchronize()
    dump_rem = [np.frombuffer(t.dump(l, b), dtype=np.uint8) for l, b in enumerate(sizes)]
    q2_found, q2_vals = query(qkeys)
    t.close()
    rec = dict(kind=kind, n0=n0, n1=n1, seed=seed, keys=keys, vals=vals.astype(np.uint64), insert_ok=ok.cpu().numpy(),
               qkeys=qkeys, q_found=q_found, q_vals=q_vals, rkeys=rkeys, remove_ok=rok.cpu().numpy(),
               q2_found=q2_found, q2_vals=q2_vals)
    for l, d in enumerate(dump_ins):
        rec[f"dump_insert_l{l}"] = d
    for l, d in enumerate(dump_rem):
        rec[f"dump_remove_l{l}"] = d
    return rec


def tcf_stats(torch):
    """Reference parallel bulk kernels on the plain-TCF workload: 2^22 slots, 1% backing,
    0.85 load, query the inserted keys and 2^22 fresh keys."""
    dev = torch.device("cuda")
    n0 = 1 << 22
    n1 = n0 // 100
    n = int(0.85 * n0)
    keys = wl.keys_without_sentinels(42, n)
    fresh = wl.keys_without_sentinels(4242, n0)
    vals = wl.values_for(keys, 2, seed=49)
    t = rc.RefTable(rc.KIND_TCF, n0, n1, 42)
    d_k = torch.from_numpy(keys.view(np.int64)).to(dev)
    d_v = torch.from_numpy(vals.view(np.int16)).to(dev)
    ok = torch.zeros(n, dtype=torch.uint8, device=dev)
    t.bulk(rc.OP_INSERT, d_k, d_v, ok)
    f = torch.zeros(n, dtype=torch.uint8, device=dev)
    t.bulk(rc.OP_QUERY, d_k, None, f)
    d_f = torch.from_numpy(fresh.view(np.int64)).to(dev)
    ff = torch.zeros(n0, dtype=torch.uint8, device=dev)
    t.bulk(rc.OP_QUERY, d_f, None, ff)
    torch.cuda.synchronize()
    okn = ok.cpu().numpy().astype(bool)
    fn = int((~f.cpu().numpy().astype(bool) & okn).sum())
    fp = int(ff.cpu().numpy().astype(bool).sum())
    t.close()
    return {"workload": "tcf 2^22 slots + 1% backing, 0.85 load, seeds 42/4242",
            "inserted": n, "insert_failures": int((~okn).sum()), "false_negatives": fn,
            "fresh_queries": n0, "false_positives": fp, "fp_rate": fp / n0}


def ht_stats(torch):
    """Reference parallel bulk kernels on the hash-table workload: 2^26 slots, bucket 8,
    20 double-hash probes, 0.9 load; queries 50% inserted / 50% absent; remove a
    seeded half; re-query.  Records order-independent checksums."""
    dev = torch.device("cuda")
    nslots = 1 << 26
    n = int(0.9 * nslots)
    keys = wl.keys_without_sentinels(43, n)
    vals = wl.values_for(keys, 8, seed=50)
    half = n // 2
    absent = wl.keys_without_sentinels(4343, half)
    qkeys = np.concatenate([keys[:half], absent])
    rem_idx = wl.fisher_yates_half(n, 77)
    t = rc.RefTable(rc.KIND_HT_DOUBLE_B8, nslots, 0, 43)
    d_k = torch.from_numpy(keys.view(np.int64)).to(dev)
    d_v = torch.from_numpy(vals.view(np.int64)).to(dev)
    ok = torch.zeros(n, dtype=torch.uint8, device=dev)
    t0 = time.time()
    t.bulk(rc.OP_INSERT, d_k, d_v, ok)
    d_q = torch.from_numpy(qkeys.view(np.int64)).to(dev)
    f = torch.zeros(len(qkeys), dtype=torch.uint8, device=dev)
    v = torch.zeros(len(qkeys), dtype=torch.int64, device=dev)
    t.bulk(rc.OP_QUERY, d_q, None, f, v)
    d_r = d_k[torch.from_numpy(rem_idx).to(dev)].contiguous()
    rok = torch.zeros(len(rem_idx), dtype=torch.uint8, device=dev)
    t.bulk(rc.OP_REMOVE, d_r, None, rok)
    f2 = torch.zeros(len(qkeys), dtype=torch.uint8, device=dev)
    v2 = torch.zeros(len(qkeys), dtype=torch.int64, device=dev)
    t.bulk(rc.OP_QUERY, d_q, None, f2, v2)
    torch.cuda.synchronize()
    el = time.time() - t0
    t.close()

    okn = ok.cpu().numpy().astype(bool)
    res = ht_exceptions(okn, vals, half, rem_idx, f.cpu().numpy(), v.cpu().numpy().view(np.uint64),
                        rok.cpu().numpy(), f2.cpu().numpy(), v2.cpu().numpy().view(np.uint64))
    res.update({"workload": "ht 2^26 slots, bucket 8, 20 double probes, 0.9 load, seeds 43/50/4343/77",
                "inserted": n, "seconds": el})
    return res


def ht_exceptions(okn, vals, half, rem_idx, found, vv, rok, found2, vv2):
    """Compare one run's query / remove results with what its own insert report
    implies (a key is present iff its insert succeeded and it was not removed;
    a present key returns its value).  Every index that disagrees is listed."""
    n_q = len(found)  # the first `half` queries are inserted keys, the rest absent
    exp_f = np.zeros(n_q, dtype=bool)
    exp_f[:half] = okn[:half]
    exp_v = np.zeros(n_q, dtype=np.uint64)
    exp_v[:half] = np.where(okn[:half], vals[:half], 0)
    q_exc = np.nonzero((found.astype(bool) != exp_f) | (vv != exp_v))[0]
    r_exc = np.nonzero(rok.astype(bool) != okn[rem_idx])[0]
    removed = np.zeros(len(okn), dtype=bool)
    removed[rem_idx[rok.astype(bool)]] = True
    exp_f2 = exp_f.copy()
    exp_f2[:half] &= ~removed[:half]
    exp_v2 = np.where(exp_f2, exp_v, 0)
    q2_exc = np.nonzero((found2.astype(bool) != exp_f2) | (vv2 != exp_v2))[0]
    return {"insert_failed": [int(i) for i in np.nonzero(~okn)[0]],
            "query_exceptions": [int(i) for i in q_exc[:1000]], "n_query_exceptions": int(len(q_exc)),
            "remove_exceptions": [int(i) for i in r_exc[:1000]], "n_remove_exceptions": int(len(r_exc)),
            "requery_exceptions": [int(i) for i in q2_exc[:1000]], "n_requery_exceptions": int(len(q2_exc)),
            "found": int(found.astype(bool).sum()), "removed": int(rok.astype(bool).sum()),
            "found_after_remove": int(found2.astype(bool).sum())}


# bucketed filters with tombstone reuse: name, kind, primary slots, backing slots, seed, #keys, key seed, tag bits
BCASES = [
    ("del_tcf", rc.KIND_DEL_TCF, 4096, 4096 // 100 + 64, 42, 3700, 1101, 16),
    ("del_tcf_small", rc.KIND_DEL_TCF_SMALL, 4096, 4096 // 100 + 64, 42, 3700, 1102, 8),
]
BOPS = ("insert", "query", "remove", "insert_delete", "insert_if_not_exists", "insert_if_not_exists_delete")


def blevels(n0: int, n1: int, tag_bits: int) -> list[int]:
    w = 4 if tag_bits == 16 else 2
    return [((n0 - 1) // 16 + 1) * 16 * w, ((n1 - 1) // 8 + 1) * 8 * w]


def run_bcase(torch, name, kind, n0, n1, seed, nkeys, kseed, bits):
    """A serial script of all six operations on a bucketed filter: insert to
    0.9 load (overflowing into the backing table), query, remove a third,
    re-add through insert_with_delete, insert_if_not_exists over a mix of
    present and absent keys, insert_if_not_exists_delete likewise.  Every
    step's results and the slot arrays after each step are recorded."""
    dev = torch.device("cuda")
    base = wl.keys_without_sentinels(kseed, nkeys)
    mask = (1 << bits) - 1
    edge = np.array([0, U64MAX, int(base[5]), 0x1234_0000_0000_0000, 0xABCD_0000_0000_0000 | mask,
                     (int(base[7]) & ~mask) | 1], dtype=np.uint64)
    keys = np.concatenate([base, edge])
    vals = wl.values_for(keys, 2, seed=kseed + 7).astype(np.uint64) & np.uint64(mask)
    fresh = wl.keys_without_sentinels(kseed + 500, 400)
    vdt, vnp = (torch.int16, np.int16) if bits == 16 else (torch.uint8, np.uint8)
    t = rc.RefTable(kind, n0, n1, seed)
    sizes = blevels(n0, n1, bits)
    rec = dict(kind=kind, n0=n0, n1=n1, seed=seed, bits=bits)

    def run(step, op, k, v=None):
        d_k = torch.from_numpy(np.ascontiguousarray(k).view(np.int64)).to(dev)
        d_v = None if v is None else torch.from_numpy(np.ascontiguousarray(v).astype(np.uint64).astype(
            np.uint16 if bits == 16 else np.uint8).view(vnp)).to(dev)
        ok = torch.zeros(len(k), dtype=torch.uint8, device=dev)
        out = torch.zeros(len(k), dtype=vdt, device=dev)
        fd = torch.zeros(len(k), dtype=torch.uint8, device=dev)
        t.bbulk(op, d_k, d_v, ok, out, fd, serial=True)
        torch.cuda.synchronize()
        o = out.cpu().numpy()
        o = (o.view(np.uint16) if bits == 16 else o).astype(np.uint64)
        rec[f"s{step}_op"] = np.array([op])
        rec[f"s{step}_keys"] = np.ascontiguousarray(k)
        rec[f"s{step}_vals"] = np.zeros(len(k), dtype=np.uint64) if v is None else np.ascontiguousarray(v).astype(np.uint64)
        rec[f"s{step}_ok"] = ok.cpu().numpy()
        rec[f"s{step}_out"] = o
        rec[f"s{step}_found"] = fd.cpu().numpy()
        for l, b in enumerate(sizes):
            rec[f"s{step}_dump_l{l}"] = np.frombuffer(t.dump(l, b), dtype=np.uint8)

    third = nkeys // 3
    mix = np.concatenate([keys[:200], fresh[:200]])
    mix2 = np.concatenate([keys[200:400], fresh[200:400]])
    mvals = (vals[:400] ^ np.uint64(0x5A)) & np.uint64(mask)
    run(0, rc.OP_INSERT, keys, vals)
    run(1, rc.OP_QUERY, np.concatenate([keys, fresh]))
    run(2, rc.OP_REMOVE, np.concatenate([keys[:third], fresh[:20]]))
    run(3, rc.OP_QUERY, np.concatenate([keys, fresh]))
    run(4, rc.OP_INSERT_DELETE, keys[: third // 2], vals[: third // 2])
    run(5, rc.OP_QUERY, np.concatenate([keys, fresh]))
    run(6, rc.OP_INSERT_IF_NOT_EXISTS, mix, mvals)
    run(7, rc.OP_INSERT_IF_NOT_EXISTS_DELETE, mix2, mvals)
    run(8, rc.OP_QUERY, np.concatenate([keys, fresh]))
    rec["steps"] = np.array([9])
    t.close()
    return rec


def btcf_stats(torch, kind, bits):
    """The reference's delete test flow (tests/src/delete_tests.cu:568-760) with
    its parallel kernels at 2^22 primary slots + 1% backing, 0.9 load: insert
    all, remove the first half, query the second half, re-add the first half
    with insert_with_delete.  Records the counts that test prints."""
    dev = torch.device("cuda")
    n0 = 1 << 22
    n1 = n0 // 100
    n = int(0.9 * (n0 + n1))
    mask = (1 << bits) - 1
    keys = wl.keys_without_sentinels(42, n)
    vals = wl.values_for(keys, 2, seed=49).astype(np.uint64) & np.uint64(mask)
    vdt, vnp = (torch.int16, np.int16) if bits == 16 else (torch.uint8, np.uint8)
    t = rc.RefTable(kind, n0, n1, 42)
    d_k = torch.from_numpy(keys.view(np.int64)).to(dev)
    d_v = torch.from_numpy(vals.astype(np.uint16 if bits == 16 else np.uint8).view(vnp)).to(dev)
    half = n // 2
    ok = torch.zeros(n, dtype=torch.uint8, device=dev)
    t.bbulk(rc.OP_INSERT, d_k, d_v, ok)
    rok = torch.zeros(half, dtype=torch.uint8, device=dev)
    t.bbulk(rc.OP_REMOVE, d_k[:half].contiguous(), None, rok)
    qf = torch.zeros(n - half, dtype=torch.uint8, device=dev)
    qv = torch.zeros(n - half, dtype=vdt, device=dev)
    t.bbulk(rc.OP_QUERY, d_k[half:].contiguous(), None, qf, qv)
    aok = torch.zeros(half, dtype=torch.uint8, device=dev)
    t.bbulk(rc.OP_INSERT_DELETE, d_k[:half].contiguous(), d_v[:half].contiguous(), aok)
    af = torch.zeros(n, dtype=torch.uint8, device=dev)
    t.bbulk(rc.OP_QUERY, d_k, None, af)
    torch.cuda.synchronize()
    okn = ok.cpu().numpy().astype(bool)
    qvn = qv.cpu().numpy()
    qvn = (qvn.view(np.uint16) if bits == 16 else qvn).astype(np.uint64)
    qfn = qf.cpu().numpy().astype(bool)
    t.close()
    return {"workload": f"bucketed filter ({bits}-bit tags) 2^22 slots + 1% backing, 0.9 load, seeds 42/49",
            "inserted": n, "insert_failures": int((~okn).sum()),
            "remove_misses": int((~rok.cpu().numpy().astype(bool)).sum()),
            "query_misses": int((~qfn & okn[half:]).sum()),
            "query_value_mismatches": int((qfn & (qvn != vals[half:])).sum()),
            "readd_failures": int((~aok.cpu().numpy().astype(bool)).sum()),
            "found_after_readd": int(af.cpu().numpy().astype(bool).sum())}


def main():
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(ROOT / "tests" / "golden"))
    ap.add_argument("--skip-stats", action="store_true")
    ap.add_argument("--bucketed-only", action="store_true", help="only the bucketed filter cases and stats")
    a = ap.parse_args()
    out = Path(a.out)
    out.mkdir(parents=True, exist_ok=True)
    for case in BCASES:
        rec = run_bcase(torch, *case)
        np.savez_compressed(out / f"ref_{case[0]}.npz", **rec)
        print(case[0], "inserted", int(rec["s0_ok"].sum()), "/", len(rec["s0_keys"]))
    if a.bucketed_only:
        if not a.skip_stats:
            bstats = {"del_tcf": btcf_stats(torch, rc.KIND_DEL_TCF, 16),
                      "del_tcf_small": btcf_stats(torch, rc.KIND_DEL_TCF_SMALL, 8)}
            (out / "ref_bucketed_stats.json").write_text(json.dumps(bstats, indent=1))
            print(json.dumps(bstats, indent=1))
        return
    for case in CASES:
        rec = run_case(torch, *case)
        np.savez_compressed(out / f"ref_{case[0]}.npz", **rec)
        print(case[0], "inserted", int(rec["insert_ok"].sum()), "/", len(rec["keys"]))
    if not a.skip_stats:
        stats = {"tcf": tcf_stats(torch), "ht": ht_stats(torch)}
        (out / "ref_stats.json").write_text(json.dumps(stats, indent=1))
        print(json.dumps(stats, indent=1))
        bstats = {"del_tcf": btcf_stats(torch, rc.KIND_DEL_TCF, 16),
                  "del_tcf_small": btcf_stats(torch, rc.KIND_DEL_TCF_SMALL, 8)}
        (out / "ref_bucketed_stats.json").write_text(json.dumps(bstats, indent=1))
        print(json.dumps(bstats, indent=1))


if __name__ == "__main__":
    main()
