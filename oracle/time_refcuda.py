"""Times the reference's own CUDA build on the secondary workloads.

Measurement infrastructure, like the rest of oracle/: nothing in the library
calls it.  It drives oracle/_ref/libpoggers_refcuda.so (the reference's
tables compiled from its own sources by oracle/Makefile, one tile per key in
the reference's launch shape) through oracle/pyrefcuda.py, on the inputs and
with the phase timers that poggers_b200.bench_configs uses for this library,
so the two JSON lines compare the same keys on the same GPU:

    python -m poggers_b200.bench_configs --config del    # this library
    python -m oracle.time_refcuda --config del           # the reference's build
    python -m poggers_b200.bench_configs --config tcf
    python -m oracle.time_refcuda --config tcf
    python -m poggers_b200.bench_configs --config 3   # 1024 TCFs: batched and per-table
    python -m oracle.time_refcuda --config 3          # the reference: one launch per table per phase
    python -m poggers_b200.bench_configs --config 5
    python -m oracle.time_refcuda --config 5          # 2^30-slot table and 2^32-slot tag-only filter

The reference's slab allocator is not run: its headers need a compile fix and
its slab code spins without a bound (offset_slab.cuh:90,169,1121,1535).
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def time_del(args):
    from oracle import pyrefcuda as rc
    from poggers_b200 import bench_configs as bc

    d = bc.del_flow(args.log2)
    ms = []
    for step in range(args.steps + 2):
        r = rc.RefTable(rc.KIND_DEL_TCF, d["n0"], d["n1"], 42)

        def run(op, k, v, fl, out=None):
            r.bbulk(op if op != 3 else rc.OP_INSERT_DELETE, k, v, fl, out)

        m = bc.del_phases(run, d)
        r.close()
        if step >= 2:
            ms.append(m)
    return {"config": "del", "impl": "reference_cuda", "keys": d["n"], "reference_cuda": bc.del_summary(ms, d)}


def time_tcf(args):
    from oracle import pyrefcuda as rc
    from poggers_b200 import bench_configs as bc

    res = {"config": "tcf", "impl": "reference_cuda"}
    for name, log2, backing, load, values in bc.TCF_WORKLOADS:
        d = bc.tcf_inputs(log2, load, values)
        n0 = 1 << log2
        kind = rc.KIND_TCF if backing else rc.KIND_TCQF
        runs = []
        for step in range(args.steps + 2):
            r = rc.RefTable(kind, n0, n0 // backing if backing else 0, 42)

            def run(op, k, v, fl):
                r.bulk(op, k, v, fl)

            out = bc.tcf_phases(run, d)
            r.close()
            if step >= 2:
                runs.append(out)
        res[name] = bc.tcf_summary(runs, d)
        del d
    return res


def _events(n):
    import torch
    return [torch.cuda.Event(enable_timing=True) for _ in range(n)]


def _clear(r, nlevels):
    """Zero a reference table's levels (its slot arrays) on the current stream."""
    import ctypes as C
    import torch
    cudart = C.CDLL("libcudart.so.12")
    cudart.cudaMemsetAsync.argtypes = [C.c_void_p, C.c_int, C.c_size_t, C.c_void_p]
    st = torch.cuda.current_stream().cuda_stream
    for l in range(nlevels):
        p, nb = r.level(l)
        cudart.cudaMemsetAsync(p, 0, nb * r.bucket_bytes(l), st)


def time_config3(args):
    """1024 TCFs (the reference's data_structs::tcf with its backing table) on
    the batched workload's tables and keys, served the only way the reference
    can: one insert launch per table, then one query launch per table."""
    import numpy as np
    import torch
    from oracle import pyrefcuda as rc
    from poggers_b200 import bench_configs as bc

    d = bc.config3_inputs(args.tables or 1024)
    offs, counts = d["offs"], d["counts"]
    dk, dv, dq = bc._dev(d["ins"]), bc._dev(d["vals"]), bc._dev(d["q"])
    N = len(d["ins"])
    ok = torch.zeros(N, dtype=torch.uint8, device="cuda")
    found = torch.zeros(N, dtype=torch.uint8, device="cuda")
    tables = [rc.RefTable(rc.KIND_TCF, int(n), int(b), sd) for n, b, sd in zip(d["sizes"], d["backing"], d["seeds"])]
    ms = []
    for rep in range(args.steps + 1):
        for r in tables:
            _clear(r, 2)
        e0, e1 = _events(2)
        e0.record()
        for i, r in enumerate(tables):
            a, b = int(offs[i]), int(offs[i + 1])
            r.bulk(0, dk[a:b], dv[a:b], ok[a:b])
        for i, r in enumerate(tables):
            a, b = int(offs[i]), int(offs[i + 1])
            r.bulk(1, dq[a:b], None, found[a:b])
        e1.record()
        torch.cuda.synchronize()
        if rep:
            ms.append(e0.elapsed_time(e1))
    okn = ok.cpu().numpy().astype(bool)
    fnd = found.cpu().numpy().astype(bool)
    fn_total = sum(int((~fnd[offs[i]:offs[i] + (offs[i + 1] - offs[i]) // 2] &
                        okn[offs[i]:offs[i] + (offs[i + 1] - offs[i]) // 2]).sum()) for i in range(len(tables)))
    for r in tables:
        r.close()
    m = float(np.median(ms))
    return {"config": 3, "impl": "reference_cuda", "keys": N, "per_table_ms": round(m, 3),
            "per_table_mops": round(2 * N / m / 1e3, 1), "insert_failures": int((~okn).sum()),
            "false_negatives": fn_total}


def time_config5(args):
    """The large plain workloads on the reference's build: the 2^30-slot uint64
    table (double hashing, bucket 8; 0.9 load, then as many Zipf(1.1) queries,
    half absent) and the 2^32-slot tag-only filter (0.9 load in 2^28-key
    chunks, then 2^30 Zipf queries), on the keys bench_configs --config 5 uses."""
    import torch
    from oracle import pyrefcuda as rc
    from poggers_b200 import bench_configs as bc
    from poggers_b200 import workload as wl

    res = {"config": 5, "impl": "reference_cuda"}
    ns = 1 << 30
    n = int(0.9 * ns)
    r = rc.RefTable(rc.KIND_HT_DOUBLE_B8, ns, 0, 43)
    k = wl.device_splitmix64(43, n)
    v = wl.device_splitmix64(50, n)
    ok = torch.zeros(n, dtype=torch.uint8, device="cuda")
    ms_ins, _ = bc._timed(lambda: r.bulk(0, k, v, ok))
    fails = int(n - ok.sum().item())
    del v
    q = bc._zipf_queries(43, n, n)
    del k
    found = torch.zeros(n, dtype=torch.uint8, device="cuda")
    qv = torch.zeros(n, dtype=torch.int64, device="cuda")
    ms_q, _ = bc._timed(lambda: r.bulk(1, q, None, found, qv))
    res["ht_2p30"] = {"inserts": n, "insert_ms": round(ms_ins, 2), "insert_mops": round(n / ms_ins / 1e3, 1),
                      "insert_failures": fails, "queries": n, "query_ms": round(ms_q, 2),
                      "query_mops": round(n / ms_q / 1e3, 1),
                      "positive_found": float(found[0::2].float().mean().item())}
    r.close()
    del q, found, qv, ok
    torch.cuda.empty_cache()
    ns = 1 << 32
    n = int(0.9 * ns)
    r = rc.RefTable(rc.KIND_TCQF, ns, 0, 42)
    chunk = 1 << 28
    fl = torch.zeros(chunk, dtype=torch.uint8, device="cuda")
    ms_ins, fails = 0.0, 0
    for s0 in range(0, n, chunk):
        c = min(chunk, n - s0)
        kk = wl.device_splitmix64(42, c, s0)
        m, _ = bc._timed(lambda: r.bulk(0, kk, None, fl[:c]))
        ms_ins += m
        fails += int(c - fl[:c].sum().item())
    del kk
    nq = 1 << 30
    ms_q, hits_pos, hits_neg = 0.0, 0, 0
    for s0 in range(0, nq, chunk):
        qq = bc._zipf_queries(42, n, chunk, qseed=11 + s0)
        m, _ = bc._timed(lambda: r.bulk(1, qq, None, fl))
        ms_q += m
        hits_pos += int(fl[0::2].sum().item())
        hits_neg += int(fl[1::2].sum().item())
    res["tcf_2p32_tag_only"] = {"inserts": n, "insert_ms": round(ms_ins, 1), "insert_mops": round(n / ms_ins / 1e3, 1),
                                "insert_failures": fails, "queries": nq, "query_ms": round(ms_q, 1),
                                "query_mops": round(nq / ms_q / 1e3, 1), "positive_found": hits_pos / (nq // 2),
                                "false_positive_rate": hits_neg / (nq // 2)}
    r.close()
    res["slab_churn"] = "not run: the reference's slab headers need a compile fix and its slab code spins without bound"
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", choices=["del", "tcf", "3", "5"], required=True)
    ap.add_argument("--tables", type=int, default=None, help="config 3: number of tables (1024)")
    ap.add_argument("--log2", type=int, default=28, help="config del: log2 of the primary slot count")
    ap.add_argument("--steps", type=int, default=5)
    a = ap.parse_args()
    from oracle import pyrefcuda as rc
    if not rc.available():
        print(json.dumps({"config": a.config, "impl": "reference_cuda",
                          "unavailable": "oracle/_ref/libpoggers_refcuda.so is not built (make -C oracle refcuda)"}))
        return
    fn = {"del": time_del, "tcf": time_tcf, "3": time_config3, "5": time_config5}[a.config]
    print(json.dumps(fn(a)))


if __name__ == "__main__":
    main()
