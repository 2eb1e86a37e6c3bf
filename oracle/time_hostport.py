"""Times the multithreaded host port of the reference's table semantics (the
CPU baseline) on the secondary workloads, on every core of this host.

Measurement infrastructure, like the rest of oracle/: nothing in the library
calls it.  The port (oracle/poggers_oracle.c, pgo_mt_bulk_*) makes the same
CAS on the same slot layout as the reference, from host threads.  Inputs are
the ones poggers_b200.bench_configs uses for the GPU:

    python -m oracle.time_hostport --config 1   # TCF 2^22 slots + 1 % backing, 0.85 load, whole workload
    python -m oracle.time_hostport --config 3   # the 1024 TCFs, whole workload, one table after another
    python -m oracle.time_hostport --config 5   # the 2^30-slot uint64 table: a sample of 2^26 inserts
                                                #   and as many queries (the table alone is 16 GiB of host memory)
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def _rate(n, el):
    return round(n / el / 1e6, 2)


def time_config1(cores):
    from oracle import pyoracle as po
    from poggers_b200 import workload as wl
    n0 = 1 << 22
    n = int(0.85 * n0)
    keys = wl.keys_without_sentinels(42, n)
    fresh = wl.keys_without_sentinels(4242, n)
    vals = (wl.values_for(keys, 2, 49).astype(np.uint64) & np.uint64(0xFFFF))
    t = po.OracleTable(1, 4, [(n0, 16, 2, 1, 0), (n0 // 100, 4, 20, 0, 0)], 42)
    t0 = time.perf_counter()
    t.insert_many(keys, vals, threads=cores)
    t.query_many(keys, threads=cores)
    t.query_many(fresh, threads=cores)
    el = time.perf_counter() - t0
    return {"workload": "TCF 2^22 slots + 1 % backing, 0.85 load: insert, query inserted, query absent",
            "mops_insert_query": _rate(3 * n, el), "seconds": round(el, 2), "sample": "the whole workload"}


def time_config3(cores):
    from oracle import pyoracle as po
    from poggers_b200 import bench_configs as bc
    d = bc.config3_inputs(1024)
    offs = d["offs"]
    tables = [po.OracleTable(1, 4, [(int(n), 16, 2, 1, 0), (int(b), 4, 20, 0, 0)], sd)
              for n, b, sd in zip(d["sizes"], d["backing"], d["seeds"])]
    vals = d["vals"].astype(np.uint64)
    t0 = time.perf_counter()
    for i, t in enumerate(tables):
        t.insert_many(d["ins"][offs[i]:offs[i + 1]], vals[offs[i]:offs[i + 1]], threads=cores)
    for i, t in enumerate(tables):
        t.query_many(d["q"][offs[i]:offs[i + 1]], threads=cores)
    el = time.perf_counter() - t0
    n = len(d["ins"])
    return {"workload": "1024 TCFs, slots log-uniform [2^12, 2^20], 1 % backing, 0.9 load; inserts then queries",
            "mops_insert_query": _rate(2 * n, el), "seconds": round(el, 2),
            "sample": "the whole workload, one table after another"}


def time_config5(cores):
    from oracle import pyoracle as po
    from poggers_b200 import workload as wl
    ns = 1 << 30
    n = 1 << 26
    keys = wl.keys_without_sentinels(43, n)
    vals = wl.values_for(keys, 8, 50)
    q = np.empty(n, dtype=np.uint64)
    q[0::2] = keys[: n // 2]
    q[1::2] = wl.keys_without_sentinels(4343, n // 2)
    t = po.OracleTable(0, 4, [(ns, 8, 20, 0, 0)], 43)
    t0 = time.perf_counter()
    t.insert_many(keys, vals, threads=cores)
    ti = time.perf_counter() - t0
    t0 = time.perf_counter()
    t.query_many(q, threads=cores)
    tq = time.perf_counter() - t0
    return {"workload": "uint64 table, 2^30 slots, bucket 8, double hashing",
            "insert_mops": _rate(n, ti), "query_mops": _rate(n, tq),
            "sample": "2^26 inserts into the empty 2^30-slot table, then 2^26 queries (half inserted)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", choices=["1", "3", "5"], required=True)
    a = ap.parse_args()
    from oracle import pyoracle as po
    cores = po.online_cores()
    fn = {"1": time_config1, "3": time_config3, "5": time_config5}[a.config]
    out = {"config": a.config, "impl": "host port (multithreaded CPU)", "cores": cores}
    out.update(fn(cores))
    print(json.dumps(out))


if __name__ == "__main__":
    main()
