"""Measurements of the secondary workloads (the headline is bench.py).

    python -m poggers_b200.bench_configs --config 1   # plain TCF, 2^22 slots
    python -m poggers_b200.bench_configs --config 3   # 1024 TCFs: batched vs per-table launches
    python -m poggers_b200.bench_configs --config 4   # served request stream vs plain per-request path
    python -m poggers_b200.bench_configs --config del # bucketed filter with deletes (2^28 slots)
    python -m poggers_b200.bench_configs --config tcf # TCF and tag-only filter, 2^22 and 2^28 slots
    python -m poggers_b200.bench_configs --config 5   # large: 2^30-slot HT, 2^32-slot tag-only TCF, slab churn, served HT
    python -m poggers_b200.bench_configs --config random  # the random-access ceilings (own kernel)
    python -m poggers_b200.bench_configs --config slab    # config 5's slab churn alone

Each prints one JSON line.  All inputs are seeded synthetic keys.  The
reference's own CUDA build is timed on the same keys by oracle/time_refcuda.py
(configs del and tcf).  hbm_frac fields are algorithmic bytes per operation x
operations per second over the measured HBM copy bandwidth.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

import poggers_b200 as pg
from poggers_b200 import workload as wl


# algorithmic bytes per operation: one minimal pass over each touched bucket
# (TCF: 8 B key + two 32 B buckets (+ a 32 B sector written); uint64 table:
# key and value + a 128 B bucket (+ a 32 B sector written); slab: an 8 B
# pointer + a 32 B bitmap sector)
ALGO_BYTES = {"tcf_insert": 104, "tcf_query": 73, "ht_insert": 176, "ht_query": 145, "slab": 40}


def hbm_frac(bytes_per_op, mops):
    """bytes_per_op x mops (millions of operations per second) over the measured
    HBM copy bandwidth (MEASURED_PEAKS.json at the repository root; 6650 GB/s
    when it is absent)."""
    from pathlib import Path
    p = Path(__file__).resolve().parent.parent / "MEASURED_PEAKS.json"
    peak = float(json.loads(p.read_text())["hbm_gbs"]) if p.exists() else 6650.0
    return round(bytes_per_op * mops * 1e6 / (peak * 1e9), 3)


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64 if a.dtype == np.uint64 else np.int16)).cuda()


def _events(n):
    import torch
    return [torch.cuda.Event(enable_timing=True) for _ in range(n)]


# ---------------------------------------------------------------- config 1
def config1(args):
    """Plain TCF: 2^22 slots of 16-bit tags (+16-bit values), buckets of 16, 1%
    backing table; insert to 0.85 load; query the inserted keys and 2^22 fresh."""
    import torch
    n0 = 1 << 22
    n = int(0.85 * n0)
    keys = wl.keys_without_sentinels(42, n)
    fresh = wl.keys_without_sentinels(4242, n0)
    vals = wl.values_for(keys, 2, 49)
    cfg = pg.data_structs.tcf(n0, n0 // 100)
    cfg.split = True
    t = pg.Table(cfg, 42)
    t.set_launch(256, 32, 0, 1)
    dk, dv, df = _dev(keys), _dev(vals), _dev(fresh)
    ok = torch.zeros(n, dtype=torch.uint8, device="cuda")
    f1 = torch.zeros(n, dtype=torch.uint8, device="cuda")
    f2 = torch.zeros(n0, dtype=torch.uint8, device="cuda")
    ins, qp, qn = [], [], []
    for step in range(args.steps + 3):
        t.clear()
        e = _events(4)
        e[0].record()
        t.bulk_insert(dk, dv, ok)
        e[1].record()
        t.bulk_query(dk, None, f1)
        e[2].record()
        t.bulk_query(df, None, f2)
        e[3].record()
        torch.cuda.synchronize()
        if step >= 3:
            ins.append(e[0].elapsed_time(e[1]))
            qp.append(e[1].elapsed_time(e[2]))
            qn.append(e[2].elapsed_time(e[3]))
    okn = ok.cpu().numpy().astype(bool)
    fn = int((~f1.cpu().numpy().astype(bool) & okn).sum())
    fp = float(f2.cpu().numpy().astype(bool).mean())
    ms = np.median(ins) + np.median(qp) + np.median(qn)
    return {"config": 1, "workload": "TCF 2^22 slots (16-bit tag+val, bucket 16) + 1% backing, 0.85 load",
            "insert_mops": round(n / np.median(ins) / 1e3, 1),
            "query_pos_mops": round(n / np.median(qp) / 1e3, 1),
            "query_neg_mops": round(n0 / np.median(qn) / 1e3, 1),
            "mops_insert_query": round((n + n + n0) / ms / 1e3, 1),
            "insert_failures": int((~okn).sum()), "false_negatives": fn, "fp_rate": fp,
            "roofline_note": "table is 16 MiB, L2-resident: bound by L2, not HBM"}


# ---------------------------------------------------------------- config 3
def config3_inputs(ntab: int, seed: int = 3):
    """1024 TCF shapes with slot counts log-uniform in [2^12, 2^20] and a 1 %
    backing level (as the plain TCF), each filled to 0.9 with its own keys; the
    queries are half the table's keys, half never inserted."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(2 ** 12), np.log(2 ** 20), ntab)).astype(np.int64)
    backing = [max(int(n) // 100, 64) for n in sizes]
    counts = (0.9 * sizes).astype(np.int64)
    keys = [wl.keys_without_sentinels(77_000 + i, int(c)) for i, c in enumerate(counts)]
    qkeys = [np.concatenate([k[: len(k) // 2], wl.keys_without_sentinels(99_000 + i, len(k) - len(k) // 2)])
             for i, k in enumerate(keys)]
    ins_all, q_all = np.concatenate(keys), np.concatenate(qkeys)
    offs = np.concatenate([[0], np.cumsum(counts)])
    vals = wl.values_for(ins_all, 2, 5)
    return {"sizes": sizes, "backing": backing, "counts": counts, "offs": offs, "ins": ins_all, "q": q_all,
            "vals": vals, "seeds": [1000 + i for i in range(ntab)]}


def config3(args):
    """1024 TCFs, slot counts log-uniform in [2^12, 2^20], each filled to 0.9.
    The batched path runs all inserts in one persistent run, then all queries
    (half inserted, half absent) in another, replayed from one captured CUDA
    graph, in the shape the autotuner picks (lanes per key x bucket size x
    blocks per SM); against 1024 per-table launches per phase on the same
    tables.  Tables are cleared (one kernel) before every timed step, outside
    the timed region, for both paths."""
    import torch
    from poggers_b200 import autotune as at
    ntab = args.tables or 1024
    d = config3_inputs(ntab)
    sizes, counts, offs = d["sizes"], d["counts"], d["offs"]
    dk, dv, dq = _dev(d["ins"]), _dev(d["vals"]), _dev(d["q"])
    N = len(d["ins"])
    ins_ops = torch.from_numpy(pg.pack_ops([(i, pg.PG_OP_INSERT, int(offs[i]), int(counts[i])) for i in range(ntab)])).cuda()
    q_ops = torch.from_numpy(pg.pack_ops([(i, pg.PG_OP_QUERY, int(offs[i]), int(counts[i])) for i in range(ntab)])).cuda()
    d_n = torch.tensor([ntab], dtype=torch.int32, device="cuda")

    def make_configs(bucket):
        return [pg.data_structs.tcf(int(n), b, bucket=bucket) for n, b in zip(sizes, d["backing"])]

    grid = {}
    if args.lanes_grid:
        grid["lanes"] = tuple(args.lanes_grid)
    if args.bucket_grid:
        grid["buckets"] = tuple(args.bucket_grid)
    if args.bps_grid:
        grid["blocks_per_sm"] = tuple(args.bps_grid)
    shape, sweep_res = at.tuned_batch_shape(make_configs, d["seeds"], ins_ops, q_ops, d_n, dk, dv, dq, **grid)
    tables = [pg.Table(c, sd) for c, sd in zip(make_configs(shape.bucket), d["seeds"])]
    ok = torch.zeros(N, dtype=torch.uint8, device="cuda")
    found = torch.zeros(N, dtype=torch.uint8, device="cuda")
    batch = pg.Batch(tables, max_ops=ntab)
    batch.set_launch(shape.block_threads, shape.blocks_per_sm, shape.lanes)

    # plain path: one launch per table per phase (each table's default launch)
    def plain():
        for i, t in enumerate(tables):
            a, b = int(offs[i]), int(offs[i + 1])
            t.bulk_insert(dk[a:b], dv[a:b], ok[a:b])
        for i, t in enumerate(tables):
            a, b = int(offs[i]), int(offs[i + 1])
            t.bulk_query(dq[a:b], None, found[a:b])

    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        batch.clear(s)
        batch.run(ins_ops, d_n, dk, dv, None, ok, None, s)
        batch.run(q_ops, d_n, dq, None, None, found, None, s)
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        batch.run(ins_ops, d_n, dk, dv, None, ok, None, s)
        batch.run(q_ops, d_n, dq, None, None, found, None, s)

    def timed(fn, reps):
        ms = []
        for _ in range(reps + 1):
            with torch.cuda.stream(s):
                batch.clear(s)
                e0, e1 = _events(2)
                e0.record(s)
                fn()
                e1.record(s)
            s.synchronize()
            ms.append(e0.elapsed_time(e1))
        return float(np.median(ms[1:]))

    plain_ms = timed(plain, args.steps)
    graph_ms = timed(g.replay, args.steps)
    with torch.cuda.stream(s):
        batch.clear(s)
        g.replay()
    s.synchronize()
    okn = ok.cpu().numpy().astype(bool)
    fnd = found.cpu().numpy().astype(bool)
    fn_total = 0
    fp_total = 0
    for i in range(ntab):
        a, b = int(offs[i]), int(offs[i + 1])
        half = (b - a) // 2
        fn_total += int((~fnd[a:a + half] & okn[a:a + half]).sum())
        fp_total += int(fnd[a + half:b].sum())
    ops = 2 * N
    del g
    batch.free()
    out = {"config": 3, "workload": f"{ntab} TCFs, slots log-uniform [2^12, 2^20] (total {int(sizes.sum())}), 1 % "
                                    "backing, 0.9 load; inserts then queries (half absent)",
           "tuned_shape": {"lanes_per_key": shape.lanes, "bucket": shape.bucket, "blocks_per_sm": shape.blocks_per_sm,
                           "block_threads": shape.block_threads},
           "keys": int(N), "plain_ms": round(plain_ms, 3), "batched_graph_ms": round(graph_ms, 3),
           "plain_mops": round(ops / plain_ms / 1e3, 1), "batched_mops": round(ops / graph_ms / 1e3, 1),
           "speedup": round(plain_ms / graph_ms, 2), "insert_failures": int((~okn).sum()),
           "false_negatives": fn_total, "fp_rate": fp_total / max(1, N - N // 2),
           "graph_kernels_per_step": 4}
    if sweep_res is not None:
        out["sweep"] = [{"lanes": r.shape.lanes, "bucket": r.shape.bucket, "blocks_per_sm": r.shape.blocks_per_sm,
                         "step_ms": round(r.step_ms, 3), "insert_failures": r.insert_failures} for r in sweep_res]
    return out


# ---------------------------------------------------------------- config 4
def _request_stream(rng, ntab, nreq, kinds, zipf_a=0.99, max_log2=16):
    w = 1.0 / np.arange(1, ntab + 1) ** zipf_a
    w /= w.sum()
    tables = rng.choice(ntab, size=nreq, p=w)
    ops = rng.choice(3, size=nreq, p=[0.3, 0.6, 0.1])
    sizes = np.floor(2 ** rng.uniform(0, max_log2, nreq)).astype(np.int64)
    return tables, ops, sizes


def config4(args):
    """Served request stream: resident tables (TCFs and uint64 double-hash tables),
    Zipf(0.99) table choice, Poisson arrivals, insert/query/delete 30/60/10,
    request sizes 2^U keys with U ~ Uniform[0, 16].  Reports served Mops/s and
    p50/p99 latency at each offered rate, and the plain per-request path."""
    import torch
    rng = np.random.default_rng(4)
    ntab = args.tables or 256
    budget = int(args.budget_gb * (1 << 30))
    per = budget // ntab
    kinds = ["tcf" if i % 2 else "ht" for i in range(ntab)]
    srv = pg.Server(hbm_budget_bytes=budget, max_wave_keys=1 << 20, max_wave_requests=4096)
    plain_tables = []
    ids = []
    for i, k in enumerate(kinds):
        if k == "ht":
            n = per // 17  # 16 B slots + 1 B fingerprints
            cfg = pg.data_structs.hash_table_64(n, bucket=8)
            cfg.fingerprints = True
        else:
            n = per // 4
            cfg = pg.data_structs.tcf(int(n * 0.95), int(n * 0.05) // 1)
        tid = srv.add_table(cfg, 500 + i)
        if tid is None:
            break
        ids.append((tid, k, n))
    nt = len(ids)
    # per-table key streams: inserts take fresh keys, queries half known / half absent, deletes known keys
    nreq = args.requests
    tsel, ops, sizes = _request_stream(rng, nt, nreq, kinds)
    fresh_pos = np.zeros(nt, dtype=np.int64)
    reqs = []
    for t, op, n in zip(tsel, ops, sizes):
        n = int(max(1, n))
        if op == 0:
            k = wl.splitmix64(900_000 + int(t), n, int(fresh_pos[t]))
            fresh_pos[t] += n
        elif op == 1:
            # half a run of keys inserted earlier (the table's key stream), half never inserted
            m = min(n // 2, int(fresh_pos[t]))
            st = int(rng.integers(0, int(fresh_pos[t]) - m + 1)) if m else 0
            pos = wl.splitmix64(900_000 + int(t), m, st)
            k = np.concatenate([pos, wl.splitmix64(5_000_000 + int(t), n - m, int(rng.integers(1 << 40)))])
        else:
            m = min(max(1, n // 4), int(fresh_pos[t]))
            st = int(rng.integers(0, int(fresh_pos[t]) - m + 1)) if m else 0
            k = wl.splitmix64(900_000 + int(t), m, st)
            if m == 0:
                continue
        reqs.append((ids[t][0], int(op), k, ids[t][1]))
    total_keys = sum(len(r[2]) for r in reqs)
    # warm-up, untimed: one single-key query per table builds the server's
    # per-class batches and loads the kernels
    one = wl.splitmix64(7, 1)
    warm = [srv.submit(tid, 1, one, None, None, None) for tid, _, _ in ids]
    for r in warm:
        srv.poll(r, wait=True)
    # each request's values (inserts) are made before the timed loop, so the
    # client submits on the arrival schedule instead of behind it
    vals_of = [wl.values_for(k, 8 if kind == "ht" else 2, 1) if op == 0 else None for _, op, k, kind in reqs]
    results = {}
    for rate in args.rates:
        tm0 = srv.timing()
        gaps = rng.exponential(1.0 / rate, len(reqs))
        arrive = np.cumsum(gaps)
        outs = [np.zeros(len(k), dtype=np.uint64 if kind == "ht" else np.uint16) if op == 1 else None
                for _, op, k, kind in reqs]
        t0 = time.perf_counter()
        rids = []
        for (tid, op, k, kind), vals, vout, at in zip(reqs, vals_of, outs, arrive):
            while time.perf_counter() - t0 < at:
                pass
            rids.append(srv.submit(tid, op, k, vals, vout, None))
        lats = [srv.poll(r, wait=True)[1] for r in rids]
        el = time.perf_counter() - t0
        tm1 = srv.timing()
        results[str(rate)] = {"offered_req_s": rate, "achieved_mops": round(total_keys / el / 1e6, 1),
                              "p50_ms": round(1e3 * float(np.percentile(lats, 50)), 3),
                              "p99_ms": round(1e3 * float(np.percentile(lats, 99)), 3),
                              "worker": {k: (round(tm1[k] - tm0[k], 4) if k.endswith("_s") else tm1[k] - tm0[k])
                                         for k in tm1}}
    waves, _ = srv.stats()
    in_use = srv.bytes_in_use()
    # plain path: the same requests one launch each, in order, from host buffers
    plain = []
    for tid, k, n in ids:
        plain.append(pg.Table(srv_config_of(k, n), 1))
    t0 = time.perf_counter()
    for tid, op, k, kind in reqs[: args.plain_requests]:
        t = plain[tid]
        dk = _dev(k)
        flags = torch.zeros(len(k), dtype=torch.uint8, device="cuda")
        if op == 0:
            vb = 8 if kind == "ht" else 2
            t.bulk_insert(dk, _dev(wl.values_for(k, vb, 1)), flags)
        elif op == 1:
            t.bulk_query(dk, None, flags)
        else:
            t.bulk_remove(dk, flags)
        flags.cpu()
    pl = time.perf_counter() - t0
    plain_keys = sum(len(r[2]) for r in reqs[: args.plain_requests])
    srv.close()
    return {"config": 4, "workload": f"{nt} resident tables ({args.budget_gb} GB budget), Zipf 0.99, Poisson arrivals, "
                                     f"insert/query/delete 30/60/10, 2^U keys U~U[0,16], {nreq} requests",
            "tables": nt, "bytes_in_use": int(in_use), "requests": nreq, "keys": int(total_keys), "waves": int(waves),
            "served": results, "plain_mops": round(plain_keys / pl / 1e6, 1),
            "plain_requests": args.plain_requests}


# ---------------------------------------------------------------- delete flow
def del_flow(log2):
    """Inputs of the reference's delete test (tests/src/delete_tests.cu:568-760)
    at 2^log2 primary slots + 1 % backing: 0.9 of the slots in seeded keys and
    16-bit values, on the device, with the halves the phases use."""
    import torch
    n0 = 1 << log2
    n1 = n0 // 100
    n = int(0.9 * (n0 + n1))
    half = n // 2
    keys = wl.keys_without_sentinels(42, n)
    vals = (wl.values_for(keys, 2, 49).astype(np.uint64) & np.uint64(0xFFFF)).astype(np.uint16)
    dk = torch.from_numpy(keys.view(np.int64)).cuda()
    dv = torch.from_numpy(vals.view(np.int16)).cuda()
    return {"n0": n0, "n1": n1, "n": n, "half": half, "dk": dk, "dv": dv, "dk1": dk[:half].contiguous(),
            "dk2": dk[half:].contiguous(), "dv1": dv[:half].contiguous(),
            "ok": torch.zeros(n, dtype=torch.uint8, device="cuda"),
            "qv": torch.zeros(n - half, dtype=torch.int16, device="cuda")}


def del_phases(run, d):
    """Insert all, remove the first half, query the second half, re-add the first
    half with insert_with_delete; run(op, keys, vals, flags[, vals_out]) with
    op 0 insert, 1 query, 2 remove, 3 insert_with_delete.  CUDA-event ms per phase."""
    import torch
    half, ok = d["half"], d["ok"]
    e = _events(5)
    e[0].record()
    run(0, d["dk"], d["dv"], ok)
    e[1].record()
    run(2, d["dk1"], None, ok[:half])
    e[2].record()
    run(1, d["dk2"], None, ok[half:], d["qv"])
    e[3].record()
    run(3, d["dk1"], d["dv1"], ok[:half])
    e[4].record()
    torch.cuda.synchronize()
    return [e[i].elapsed_time(e[i + 1]) for i in range(4)]


def del_summary(ms, d):
    med = np.median(np.array(ms), axis=0)
    n, half = d["n"], d["half"]
    units = [n, half, n - half, half]
    names = ["insert", "remove", "query", "insert_with_delete"]
    out = {f"{k}_mops": round(u / m / 1e3, 1) for k, u, m in zip(names, units, med)}
    out["total_mops"] = round(sum(units) / med.sum() / 1e3, 1)
    out["ms"] = [round(float(x), 3) for x in med]
    return out


def config_del(args):
    """The reference's delete test on the bucketed filter with tombstone reuse:
    2^log2 primary slots + 1 % backing, 16-bit tags.  Each phase is timed with
    CUDA events, at 1 and 4 lanes per key.  (oracle/time_refcuda.py times the
    reference's own CUDA build on the same keys.)"""
    d = del_flow(args.log2)
    res = {"config": "del", "workload": f"bucketed filter, 16-bit tags: 2^{args.log2} slots (16/bucket) + 1% "
                                       f"backing (8/bucket, linear), 0.9 load; insert, remove 1/2, query 1/2, "
                                       f"re-add 1/2", "keys": d["n"]}
    for lanes in (1, 4):
        t = pg.Table(pg.data_structs.del_tcf(d["n0"], d["n1"]), 42)
        t.set_launch(256, 32, 0, lanes)

        def run(op, k, v, fl, out=None):
            if op == 0:
                t.bulk_insert(k, v, fl)
            elif op == 1:
                t.bulk_query(k, out, fl)
            elif op == 2:
                t.bulk_remove(k, fl)
            else:
                t.bulk_insert_with_delete(k, v, fl)

        ms = []
        for step in range(args.steps + 2):
            t.clear()
            m = del_phases(run, d)
            if step >= 2:
                ms.append(m)
        res[f"ours_lanes{lanes}"] = del_summary(ms, d)
        del t
    return res


# ---------------------------------------------------------------- config tcf
# The two-choice filters of the reference's data_structs (tcf.cuh:30, with a
# 1 % backing table; and the tag-only filter of bucket_speed_tests.cu:108)
# at an L2-resident and an HBM-resident size.
TCF_WORKLOADS = [
    # name, log2 slots, backing fraction, load, values
    ("tcf_2p22", 22, 100, 0.85, True),
    ("tcf_2p28", 28, 100, 0.85, True),
    ("tag_only_2p28", 28, 0, 0.9, False),
]


def tcf_inputs(log2, load, values):
    import torch
    n = int(load * (1 << log2))
    keys = wl.keys_without_sentinels(42, n)
    fresh = wl.keys_without_sentinels(4242, n)
    vals = (wl.values_for(keys, 2, 49).astype(np.uint64) & np.uint64(0xFFFF)).astype(np.uint16)
    return {"n": n, "dk": torch.from_numpy(keys.view(np.int64)).cuda(),
            "df": torch.from_numpy(fresh.view(np.int64)).cuda(),
            "dv": torch.from_numpy(vals.view(np.int16)).cuda() if values else None,
            "ok": torch.zeros(n, dtype=torch.uint8, device="cuda"),
            "found": torch.zeros(n, dtype=torch.uint8, device="cuda")}


def tcf_phases(run, d):
    """Insert all keys, query them, query as many absent keys; run(op, keys,
    vals, flags) with op 0 insert, 1 query.  Returns CUDA-event ms per phase and
    the failures, false negatives and false positives of the run."""
    import torch
    e = _events(4)
    e[0].record()
    run(0, d["dk"], d["dv"], d["ok"])
    e[1].record()
    run(1, d["dk"], None, d["found"])
    e[2].record()
    fn = int(((d["found"] == 0) & (d["ok"] == 1)).sum().item())
    e2 = _events(2)
    e2[0].record()
    run(1, d["df"], None, d["found"])
    e2[1].record()
    torch.cuda.synchronize()
    return ([e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2]), e2[0].elapsed_time(e2[1])],
            int((d["ok"] == 0).sum().item()), fn, int(d["found"].sum().item()))


def tcf_summary(runs, d):
    ms = np.median(np.array([r[0] for r in runs]).reshape(len(runs), -1), axis=0)
    n = d["n"]
    mops = [n / m / 1e3 for m in ms]
    return {"insert_mops": round(mops[0], 1), "query_positive_mops": round(mops[1], 1),
            "query_negative_mops": round(mops[2], 1),
            "insert_query_mops": round(3 * n / ms.sum() / 1e3, 1), "ms": [round(float(x), 3) for x in ms],
            "insert_failures": runs[-1][1], "false_negatives": runs[-1][2], "fp_rate": runs[-1][3] / n,
            "hbm_frac": {"insert": hbm_frac(ALGO_BYTES["tcf_insert"], mops[0]),
                         "query_positive": hbm_frac(ALGO_BYTES["tcf_query"], mops[1]),
                         "query_negative": hbm_frac(ALGO_BYTES["tcf_query"], mops[2])}}


def config_tcf(args):
    """The TCF and the tag-only filter: insert to their load, query the keys,
    query as many absent keys (default launch shape).  (oracle/time_refcuda.py
    times the reference's own CUDA build on the same keys.)"""
    res = {"config": "tcf", "workload": "TCF (16-bit tags + values, 16-slot buckets, 1 % backing) at 0.85 load "
                                        "and the tag-only filter at 0.9 load; insert, query inserted, query absent"}
    for name, log2, backing, load, values in TCF_WORKLOADS:
        if args.only and name not in args.only:
            continue
        if args.tcf_log2:  # a smaller table of the same kind (profiling captures)
            log2 = args.tcf_log2
            name = f"{name}_at_2p{log2}"
        d = tcf_inputs(log2, load, values)
        n0 = 1 << log2
        cfg = pg.data_structs.tcf(n0, n0 // backing) if backing else pg.data_structs.tcqf(n0)
        t = pg.Table(cfg, 42)

        def run(op, k, v, fl):
            if op == 0:
                t.bulk_insert(k, v, fl)
            else:
                t.bulk_query(k, None, fl)

        runs = []
        warm = 2 if args.steps > 0 else 1  # --steps 0: one warm-up and one measured run (profiling captures)
        for step in range(max(args.steps, 1) + warm):
            t.clear()
            r = tcf_phases(run, d)
            if step >= warm:
                runs.append(r)
        res[name] = tcf_summary(runs, d)
        del t, d
    return res


def _timed(fn):
    import torch
    e = _events(2)
    e[0].record()
    r = fn()
    e[1].record()
    torch.cuda.synchronize()
    return e[0].elapsed_time(e[1]), r


def _zipf_queries(seed, n_inserted, count, a=1.1, qseed=7):
    """Half Zipf(a)-ranked keys of the inserted stream, half never-inserted keys
    (interleaved), generated on the device."""
    import torch
    npos, nneg = (count + 1) // 2, count // 2  # even positions positive, odd positions absent
    ranks = wl.device_zipf_ranks(n_inserted, npos, a, qseed)
    q = torch.empty(count, dtype=torch.int64, device="cuda")
    q[0::2] = _splitmix_at(seed, ranks)
    del ranks
    q[1::2] = wl.device_splitmix64(seed ^ 0x5A5A5A5A, nneg, 0)
    return q


def _splitmix_at(seed, idx):
    """splitmix64(seed) at the given int64 indices (device)."""
    import torch

    def lsr(x, s):
        return torch.bitwise_right_shift(x, s) & ((1 << (64 - s)) - 1)

    z = (idx + 1) * wl._s64(int(wl.GAMMA)) + wl._s64(seed)
    z = (z ^ lsr(z, 30)) * wl._s64(int(wl.M1))
    z = (z ^ lsr(z, 27)) * wl._s64(int(wl.M2))
    z = z ^ lsr(z, 31)
    z = torch.where(z == 0, torch.ones_like(z), z)
    return torch.where(z == -1, torch.full_like(z, -2), z)


def config5(args):
    """Large workloads: a 2^30-slot uint64 table (16 GiB + 1 GiB fingerprints) and
    a 2^32-slot tag-only TCF (8 GiB), each filled to 0.9 and queried with as many
    Zipf(1.1) keys (half inserted, half absent); slab churn over 2^24
    allocations of log-uniform sizes in [16, 4096] B (9 power-of-two classes):
    malloc all, free a seeded random half, malloc it again; then the same
    workload through the serving loop (config5_served).  Plain launches are
    timed with CUDA events; the served path by the host clock around submit /
    poll."""
    import torch
    res = {"config": 5}
    # ---- uint64 table, 2^30 slots
    ns = 1 << 30
    n = int(0.9 * ns)
    cfg = pg.data_structs.hash_table_64(ns, bucket=8)
    cfg.fingerprints = True
    t = pg.Table(cfg, 43)
    t.set_launch(256, 32, 0, 1)
    # the region sort's scratch (about 20 bytes per key) is set up before the
    # timed call, like the table itself
    t.reserve_insert_scratch(n)
    torch.cuda.synchronize()
    k = wl.device_splitmix64(43, n)
    v = wl.device_splitmix64(50, n)
    ok = torch.zeros(n, dtype=torch.uint8, device="cuda")
    ms_ins, _ = _timed(lambda: t.bulk_insert(k, v, ok))
    fails = int(n - ok.sum().item())
    del v
    q = _zipf_queries(43, n, n)
    del k
    found = torch.zeros(n, dtype=torch.uint8, device="cuda")
    qv = torch.zeros(n, dtype=torch.int64, device="cuda")
    ms_q, _ = _timed(lambda: t.bulk_query(q, qv, found))
    pos_found = float(found[0::2].float().mean().item())
    neg_found = float(found[1::2].float().mean().item())
    res["ht_2p30"] = {"slots": ns, "inserts": n, "insert_ms": round(ms_ins, 2), "insert_mops": round(n / ms_ins / 1e3, 1),
                      "insert_failures": fails, "queries": n, "query_ms": round(ms_q, 2),
                      "query_mops": round(n / ms_q / 1e3, 1), "positive_found": pos_found,
                      "negative_found": neg_found, "table_bytes": t.host_bytes_in_use()}
    del q, found, qv, ok, t
    torch.cuda.empty_cache()
    # ---- tag-only TCF, 2^32 slots, in chunks of 2^28 keys
    ns = 1 << 32
    n = int(0.9 * ns)
    t = pg.Table(pg.data_structs.tcqf(ns), 42)
    t.set_launch(256, 32, 0, 1)
    chunk = 1 << 28
    fails = torch.zeros(1, dtype=torch.int64, device="cuda")
    ms_ins = 0.0
    for s0 in range(0, n, chunk):
        c = min(chunk, n - s0)
        kk = wl.device_splitmix64(42, c, s0)
        m, _ = _timed(lambda: t.bulk_insert(kk, None, None, fails))
        ms_ins += m
    del kk
    nq = 1 << 30
    ms_q = 0.0
    hits_pos = hits_neg = 0
    for s0 in range(0, nq, chunk):
        qq = _zipf_queries(42, n, chunk, qseed=11 + s0)
        f = torch.zeros(chunk, dtype=torch.uint8, device="cuda")
        m, _ = _timed(lambda: t.bulk_query(qq, None, f))
        ms_q += m
        hits_pos += int(f[0::2].sum().item())
        hits_neg += int(f[1::2].sum().item())
    res["tcf_2p32_tag_only"] = {"slots": ns, "inserts": n, "insert_ms": round(ms_ins, 1),
                                "insert_mops": round(n / ms_ins / 1e3, 1), "insert_failures": int(fails.item()),
                                "queries": nq, "query_ms": round(ms_q, 1), "query_mops": round(nq / ms_q / 1e3, 1),
                                "positive_found": hits_pos / (nq // 2), "false_positive_rate": hits_neg / (nq // 2),
                                "table_bytes": t.host_bytes_in_use()}
    del qq, f, t
    torch.cuda.empty_cache()
    # ---- slab churn
    res["slab_churn"] = slab_churn(1 << 24)
    # ---- served: the same workload through the serving loop, from host buffers
    res["served"] = config5_served(args)
    ht, tcf, slab = res["ht_2p30"], res["tcf_2p32_tag_only"], res["slab_churn"]
    ht["hbm_frac"] = {"insert": hbm_frac(ALGO_BYTES["ht_insert"], ht["insert_mops"]),
                      "query": hbm_frac(ALGO_BYTES["ht_query"], ht["query_mops"])}
    tcf["hbm_frac"] = {"insert": hbm_frac(ALGO_BYTES["tcf_insert"], tcf["insert_mops"]),
                       "query": hbm_frac(ALGO_BYTES["tcf_query"], tcf["query_mops"])}
    slab["hbm_frac"] = {k: hbm_frac(ALGO_BYTES["slab"], slab[k + "_mops"]) for k in ("malloc", "free", "remalloc")}
    return res


def _host(t):
    """A device int64 tensor as a host uint64 array."""
    return t.cpu().numpy().view(np.uint64)


def _serve_phase(srv, submit_all):
    """Submit every request of a phase at once, then collect them; returns the
    phase's wall time and the requests' latencies and counts."""
    t0 = time.perf_counter()
    rids = submit_all()
    got = [srv.poll(r, wait=True) for r in rids]
    el = time.perf_counter() - t0
    return el, [g[1] for g in got], [g[0] for g in got]


def _lat(lats):
    return {"p50_ms": round(1e3 * float(np.percentile(lats, 50)), 2),
            "p99_ms": round(1e3 * float(np.percentile(lats, 99)), 2)}


def slab_churn(na: int):
    """na allocations with sizes log-uniform in [16, 4096) B over the 9
    power-of-two size classes (one pool each, 5 % spare): malloc all, free a
    seeded random half, malloc that half again; CUDA-event timed."""
    import torch
    rng = np.random.default_rng(5)
    sizes = np.floor(2.0 ** rng.uniform(4, 12, na)).astype(np.uint32)
    classes = [16 << i for i in range(9)]
    cls = np.searchsorted(np.array(classes), sizes)
    counts = np.bincount(cls, minlength=9)
    allocs = [int(c * 1.05) + 4096 for c in counts]
    ss = pg.allocators.size_class_set(classes, allocs)
    d_sizes = torch.from_numpy(sizes.view(np.int32)).cuda()
    ptrs = torch.zeros(na, dtype=torch.int64, device="cuda")
    fc = torch.zeros(1, dtype=torch.int64, device="cuda")
    ms_m, _ = _timed(lambda: ss.bulk_malloc(d_sizes, ptrs, fc))
    half = torch.from_numpy(wl.fisher_yates_half(na, 77)).cuda()
    hp = ptrs[half].contiguous()
    bad = torch.zeros(1, dtype=torch.int64, device="cuda")
    ms_f, _ = _timed(lambda: ss.bulk_free(hp, bad))
    hs = d_sizes[half].contiguous()
    hp2 = torch.zeros_like(hp)
    fc2 = torch.zeros(1, dtype=torch.int64, device="cuda")
    ms_m2, _ = _timed(lambda: ss.bulk_malloc(hs, hp2, fc2))
    out = {"allocations": na, "classes": classes, "malloc_ms": round(ms_m, 2),
           "malloc_mops": round(na / ms_m / 1e3, 1), "free_ms": round(ms_f, 2),
           "free_mops": round(len(half) / ms_f / 1e3, 1), "remalloc_ms": round(ms_m2, 2),
           "remalloc_mops": round(len(half) / ms_m2 / 1e3, 1), "malloc_failures": int(fc.item()),
           "free_rejected": int(bad.item()), "remalloc_failures": int(fc2.item()),
           "pool_bytes": int(sum(ss.class_report(c)["pool_bytes"] for c in range(9)))}
    del ss, ptrs, hp, hp2
    torch.cuda.empty_cache()
    return out


def config_slab(args):
    """Config 5's slab churn alone (--allocs allocations)."""
    return {"config": "slab", "slab_churn": slab_churn(args.allocs)}


def config5_served(args):
    """Config 5 through the serving loop: the 2^30-slot uint64 table and the
    2^32-slot tag-only filter resident in one server beside the 9-class slab
    set, and the plain workload's keys, values, Zipf(1.1) queries and slab
    churn submitted from host buffers in requests of 2^22 keys (2^20 slab
    requests), phase by phase; every phase's requests are submitted at once
    and collected, so the waves run back to back.  Keys are made on the device
    and copied to host memory outside the timed phases (host generation would
    be slower than the server)."""
    import torch
    req = 1 << 22
    out = {"request_keys": req}
    srv = pg.Server(hbm_budget_bytes=60 << 30, max_wave_keys=1 << 22, max_wave_requests=64)
    ns = 1 << 30
    n = int(0.9 * ns)
    cfg = pg.data_structs.hash_table_64(ns, bucket=8)
    cfg.fingerprints = True
    tid = srv.add_table(cfg, 43)
    keys, vals = _host(wl.device_splitmix64(43, n)), _host(wl.device_splitmix64(50, n))
    el, lat, cnt = _serve_phase(srv, lambda: [srv.submit(tid, pg.PG_OP_INSERT, keys[s:s + req], vals[s:s + req])
                                              for s in range(0, n, req)])
    out["ht_2p30_insert"] = {"keys": n, "mops_e2e": round(n / el / 1e6, 1), "failures": int(sum(cnt)), **_lat(lat)}
    del keys, vals
    q = _host(_zipf_queries(43, n, n))
    vout = np.zeros(n, dtype=np.uint64)
    el, lat, cnt = _serve_phase(srv, lambda: [srv.submit(tid, pg.PG_OP_QUERY, q[s:s + req], None, vout[s:s + req])
                                              for s in range(0, n, req)])
    out["ht_2p30_query"] = {"keys": n, "mops_e2e": round(n / el / 1e6, 1), "hits": int(sum(cnt)), **_lat(lat)}
    del q, vout
    torch.cuda.empty_cache()
    ns = 1 << 32
    n = int(0.9 * ns)
    fid = srv.add_table(pg.data_structs.tcqf(ns), 42)
    keys = np.empty(n, dtype=np.uint64)
    for s0 in range(0, n, 1 << 28):
        c = min(1 << 28, n - s0)
        keys[s0:s0 + c] = _host(wl.device_splitmix64(42, c, s0))
    el, lat, cnt = _serve_phase(srv, lambda: [srv.submit(fid, pg.PG_OP_INSERT, keys[s:s + req])
                                              for s in range(0, n, req)])
    out["tcf_2p32_insert"] = {"keys": n, "mops_e2e": round(n / el / 1e6, 1), "failures": int(sum(cnt)), **_lat(lat)}
    del keys
    nq = 1 << 30
    q = np.empty(nq, dtype=np.uint64)
    for s0 in range(0, nq, 1 << 28):
        q[s0:s0 + (1 << 28)] = _host(_zipf_queries(42, n, 1 << 28, qseed=11 + s0))
    el, lat, cnt = _serve_phase(srv, lambda: [srv.submit(fid, pg.PG_OP_QUERY, q[s:s + req])
                                              for s in range(0, nq, req)])
    out["tcf_2p32_query"] = {"keys": nq, "mops_e2e": round(nq / el / 1e6, 1), "hits": int(sum(cnt)), **_lat(lat)}
    del q
    # slab churn: malloc all, free a seeded random half, malloc that half again
    rng = np.random.default_rng(5)
    na = 1 << 24
    sizes = np.floor(2.0 ** rng.uniform(4, 12, na)).astype(np.uint32)
    classes = [16 << i for i in range(9)]
    counts = np.bincount(np.searchsorted(np.array(classes), sizes), minlength=9)
    sid = srv.add_slab_set(classes, [int(c * 1.05) + 4096 for c in counts])
    sreq = 1 << 20
    ptrs = np.zeros(na, dtype=np.uint64)
    el, lat, cnt = _serve_phase(srv, lambda: [srv.submit_slab(sid, pg.PG_OP_MALLOC, sizes[s:s + sreq], ptrs[s:s + sreq])
                                              for s in range(0, na, sreq)])
    out["slab_malloc"] = {"allocations": na, "mops_e2e": round(na / el / 1e6, 1), "failures": int(sum(cnt)),
                          **_lat(lat)}
    half = wl.fisher_yates_half(na, 77)
    hp, hs = ptrs[half].copy(), sizes[half].copy()
    el, lat, cnt = _serve_phase(srv, lambda: [srv.submit_slab(sid, pg.PG_OP_FREE, hp[s:s + sreq])
                                              for s in range(0, len(hp), sreq)])
    out["slab_free"] = {"frees": len(hp), "mops_e2e": round(len(hp) / el / 1e6, 1), "refused": int(sum(cnt)),
                        **_lat(lat)}
    hp2 = np.zeros(len(hs), dtype=np.uint64)
    el, lat, cnt = _serve_phase(srv, lambda: [srv.submit_slab(sid, pg.PG_OP_MALLOC, hs[s:s + sreq], hp2[s:s + sreq])
                                              for s in range(0, len(hs), sreq)])
    out["slab_remalloc"] = {"allocations": len(hs), "mops_e2e": round(len(hs) / el / 1e6, 1),
                            "failures": int(sum(cnt)), **_lat(lat)}
    out["bytes_in_use"] = int(srv.bytes_in_use())
    out["note"] = ("host buffers in and out through the server's pinned staging and PCIe; the plain figures "
                   "are device-resident bulk launches")
    srv.close()
    return out


def srv_config_of(kind, n):
    if kind == "ht":
        cfg = pg.data_structs.hash_table_64(n, bucket=8)
        cfg.fingerprints = True
        return cfg
    return pg.data_structs.tcf(int(n * 0.95), int(n * 0.05))


def config_random(args):
    """The GPU's random-access ceilings, the filters' regime, measured by this
    library's own kernel (pg_diag_random_access): random 32-byte sectors, random
    64-byte pairs of sectors, a sector read followed by a CAS on it (an insert's
    claim), the same plus a 2-byte store into the next sector (a split filter
    bucket's insert: tag claimed, then its value written), and atomic adds with
    no return (write-only read-modify-writes), at
    the filters' table sizes (512 MiB = the tags of a 2^28-slot TCF, 1 GiB =
    its tags and values, 8 GiB = a 2^32-slot tag-only filter).  Several
    accesses are in flight per thread; CUDA-event timed, best of 5 after a
    warm-up, over 4 and 8 blocks of 256 threads per SM.  A 32 MiB buffer,
    which stays in L2, gives the L2's own rates for the same accesses (the
    uint64 table's fingerprint words live there)."""
    import torch
    modes = {"read32": pg.PG_DIAG_READ32, "read64": pg.PG_DIAG_READ64, "read32_cas": pg.PG_DIAG_READ32_CAS,
             "red32": pg.PG_DIAG_RED32, "read32_cas_next": pg.PG_DIAG_READ32_CAS_NEXT}
    if args.calibrate:
        # one launch per kind over a 1 GiB and a 32 MiB buffer (for an ncu capture of DRAM and L2 traffic)
        done = {}
        for lg in (30, 25):
            buf = torch.zeros(1 << lg, dtype=torch.uint8, device="cuda")
            for name, mode in modes.items():
                done[f"{(1 << lg) >> 20}MiB_{name}"] = pg.diag_random_access(buf, mode, 1 << 26, seed=mode + 1,
                                                                               blocks_per_sm=8)
                torch.cuda.synchronize()
            del buf
        return {"config": "random", "calibrate": done}
    sectors = {"read32": 1, "read64": 2, "read32_cas": 1, "red32": 1, "read32_cas_next": 1}
    out = {"config": "random", "note": "G accesses/s; sector_g_per_s counts the 32-byte sectors read per access"}
    sink = torch.zeros(1, dtype=torch.int64, device="cuda")
    for log2_bytes in (25, 29, 30, 33):  # 32 MiB stays in L2: the L2's own rates
        buf = torch.zeros(1 << log2_bytes, dtype=torch.uint8, device="cuda")
        res = {}
        for name, mode in modes.items():
            best = None
            for bps in (4, 8):
                for rep in range(6):
                    e = _events(2)
                    e[0].record()
                    done = pg.diag_random_access(buf, mode, 1 << 27, seed=rep + 1, blocks_per_sm=bps, sink=sink)
                    e[1].record()
                    torch.cuda.synchronize()
                    if rep == 0:
                        continue
                    rate = done / e[0].elapsed_time(e[1]) / 1e6
                    if best is None or rate > best[0]:
                        best = (rate, bps)
            res[name] = {"g_per_s": round(best[0], 2), "sector_g_per_s": round(best[0] * sectors[name], 2),
                         "sector_gbs": round(best[0] * sectors[name] * 32, 1), "blocks_per_sm": best[1]}
        out[f"buffer_{(1 << log2_bytes) >> 20}MiB"] = res
        del buf
        torch.cuda.empty_cache()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", choices=["1", "3", "4", "5", "del", "tcf", "random", "slab"], required=True)
    ap.add_argument("--allocs", type=int, default=1 << 24, help="config slab: allocations")
    ap.add_argument("--calibrate", action="store_true", help="config random: one launch per kind (ncu captures)")
    ap.add_argument("--log2", type=int, default=28, help="config del: log2 of the primary slot count")
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--only", nargs="+", default=None, help="config tcf: run only these workloads")
    ap.add_argument("--tcf-log2", type=int, default=0, help="config tcf: log2 slots instead of each workload's own")
    ap.add_argument("--tables", type=int, default=None, help="tables (config 3: 1024, config 4: 256)")
    ap.add_argument("--lanes-grid", type=int, nargs="+", default=None, help="config 3: the tuner's lanes per key")
    ap.add_argument("--bucket-grid", type=int, nargs="+", default=None, help="config 3: the tuner's bucket sizes")
    ap.add_argument("--bps-grid", type=int, nargs="+", default=None, help="config 3: the tuner's blocks per SM")
    ap.add_argument("--bucket", type=int, default=16)
    ap.add_argument("--lanes", type=int, default=1)
    ap.add_argument("--blocks-per-sm", type=int, default=8)
    ap.add_argument("--budget-gb", type=float, default=40.0)
    ap.add_argument("--requests", type=int, default=4000)
    ap.add_argument("--plain-requests", type=int, default=1000)
    ap.add_argument("--rates", type=float, nargs="+", default=[2000.0, 8000.0, 32000.0, 64000.0, 96000.0, 128000.0])
    a = ap.parse_args()
    import torch
    torch.cuda.init()
    fn = {"1": config1, "3": config3, "4": config4, "5": config5, "del": config_del, "tcf": config_tcf,
          "random": config_random, "slab": config_slab}[a.config]
    print(json.dumps(fn(a)))


if __name__ == "__main__":
    main()
