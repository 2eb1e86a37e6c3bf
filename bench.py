#!/usr/bin/env python
"""Benchmark: Mops/s insert+query at 0.9 load on the modular uint64 hash table.

Workload (one step): clear a 2^26-slot uint64->uint64 table (bucket 8, tile 4,
20 double-hash probes, 1 GiB), bulk-insert 0.9 * 2^26 = 60,397,977 seeded keys,
then bulk-query 60,397,976 keys of which half were inserted and half never
were.  value = (inserts + queries) / elapsed.  The table (1 GiB) is larger than
the 126 MB L2, so every step runs out of HBM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl {ours,reference}]
                    [--ref-target {cpu,cuda}]

--impl reference times the reference algorithm on the host cores (the
multithreaded port of the reference's table semantics in oracle/, one whole
workload per step), or with
--ref-target cuda the reference's own CUDA build (oracle/_ref) on this GPU.
Under torchrun every rank runs its own independent table (weak scaling, no
data-path collective); rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

NSLOTS = 1 << 26
BUCKET = 8
TILE = 4          # the reference's Partition_Size for this table (semantics)
LANES = 2         # lanes per key the kernels use (launch shape; results do not depend on it)
LAYOUT = "fingerprints"  # reference {key,val} slots + an L2-resident fingerprint byte per slot
BLOCK_THREADS = 256
BLOCKS_PER_SM = 32
PROBES = 20
LOAD = 0.9
SEED = 43
ALGO_BYTES = {"insert": 176, "query": 145}  # bytes per op: 16 key+val + 128 bucket + 32 write / 8 + 128 + 8 + 1
METRIC = "Mops/s insert+query at 0.9 load"
WORKLOAD = ("ht_u64: uint64->uint64 modular hash table, 2^26 slots, bucket 8, tile 4, 20 double-hash probes; "
            "insert 0.9*2^26 keys, then query as many (50% inserted, 50% absent)")


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_summary():
    """Per-launch DRAM bytes of the two kernels from the committed ncu summary."""
    p = ROOT / "profiles" / "ht_traffic.json"
    if p.exists():
        return json.loads(p.read_text())
    return None


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.idx)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def make_inputs():
    from poggers_b200 import workload as wl

    n = int(LOAD * NSLOTS)
    keys = wl.keys_without_sentinels(SEED, n)
    vals = wl.values_for(keys, 8, 50)
    half = n // 2
    qkeys = np.concatenate([keys[:half], wl.keys_without_sentinels(4343, n - half)])
    return keys, vals, qkeys


# ------------------------------------------------------------------ our arm
def run_ours(args, rank, world):
    import torch
    import poggers_b200 as pg

    dev = torch.device("cuda", torch.cuda.current_device())
    keys, vals, qkeys = make_inputs()
    n, nq = len(keys), len(qkeys)
    d_keys = torch.from_numpy(keys.view(np.int64)).to(dev)
    d_vals = torch.from_numpy(vals.view(np.int64)).to(dev)
    d_q = torch.from_numpy(qkeys.view(np.int64)).to(dev)
    ok = torch.empty(n, dtype=torch.uint8, device=dev)
    found = torch.empty(nq, dtype=torch.uint8, device=dev)
    qv = torch.empty(nq, dtype=torch.int64, device=dev)
    cfg = pg.data_structs.hash_table_64(NSLOTS, tile=TILE, bucket=BUCKET, max_probes=PROBES)
    cfg.split = args.layout == "split"
    cfg.fingerprints = args.layout == "fingerprints"
    table = pg.Table(cfg, SEED)
    table.set_launch(BLOCK_THREADS, BLOCKS_PER_SM, 0, LANES)
    table.set_partitioned_insert(args.insert_order == "region")
    stream = torch.cuda.current_stream()

    def step(ev=None):
        table.clear(stream)
        if ev:
            ev[0].record(stream)
        table.bulk_insert(d_keys, d_vals, ok, None, stream)
        if ev:
            ev[1].record(stream)
        table.bulk_query(d_q, qv, found, None, stream)
        if ev:
            ev[2].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    sampler = ClockSampler(dev.index) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    barrier(world)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for k in range(args.steps):
        step(evs[k])
    t1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop() if sampler else None
    ms = t0.elapsed_time(t1)
    ms_max = allreduce_max(ms, world)
    ins_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in evs)
    qry_ms = statistics.mean(e[1].elapsed_time(e[2]) for e in evs)

    # consistency of the last step: every inserted key of the positive half is found
    okn = ok.cpu().numpy().astype(bool)
    fn = found.cpu().numpy().astype(bool)
    qvn = qv.cpu().numpy().view(np.uint64)
    half = n // 2
    assert (fn[:half] == okn[:half]).all() and not fn[half:].any(), "query results disagree with the insert report"
    assert (qvn[:half][okn[:half]] == vals[:half][okn[:half]]).all(), "a found key returned another value"

    # one extra untimed pass for the remove rate
    rem = torch.from_numpy(keys[: n // 2].view(np.int64)).to(dev)
    rok = torch.empty(len(rem), dtype=torch.uint8, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    table.bulk_remove(rem, rok, None, stream)
    e1.record(stream)
    torch.cuda.synchronize()
    rem_ms = e0.elapsed_time(e1)

    e2e = None if args.no_e2e else run_e2e(args, table, keys, vals, qkeys, dev, world)

    # per step: the insert kernel (after the run bases and scatter kernels, and
    # followed by the pass for keys that missed their run, when the batch is
    # region-ordered) and the query kernel; clears are memsets
    ordered = args.insert_order == "region" and n >= (1 << 20) and NSLOTS * 16 >= (64 << 20)
    launches_per_step = (4 if ordered else 1) + 1
    ops = (n + nq) * args.steps * world
    value = ops / (ms_max / 1e3) / 1e6
    peak, peak_kind = peaks()
    dom = "insert" if ins_ms >= qry_ms else "query"
    dom_ms = max(ins_ms, qry_ms)
    dom_units = n if dom == "insert" else nq
    achieved = ALGO_BYTES[dom] * dom_units / (dom_ms / 1e3) / 1e9
    tr = traffic_summary()
    traffic = None
    # the summary's bytes are per launch of its own key count, for the fingerprint
    # layout with region-ordered inserts; they scale with the keys of a launch
    if tr and dom in tr and args.layout == "fingerprints" and args.insert_order == "region":
        traffic = round(tr[dom]["dram_bytes_per_launch"] * dom_units / tr["keys_per_launch"])
    out = {
        "metric": METRIC, "value": round(value, 1), "unit": "Mops/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded splitmix64 keys)",
        "config": {"workload": WORKLOAD, "slots": NSLOTS, "inserts": n, "queries": nq,
                   "launch": {"lanes_per_key": 1 if args.layout == "fingerprints" else LANES,
                              "block_threads": BLOCK_THREADS, "blocks_per_sm": BLOCKS_PER_SM,
                              "bucket_layout": args.layout, "insert_order": args.insert_order},
                   "parallelism": f"independent table per GPU x{world}",
                   "l2": f"inputs larger than L2 ({NSLOTS * 16 >> 20} MiB table, 126 MB L2)"},
        "roofline": {"bound": "hbm", "kernel": f"bulk_{dom}", "achieved": round(achieved, 1),
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": traffic, "algo_bytes_per_op": ALGO_BYTES[dom], "units_per_launch": dom_units},
        "kernels": {"insert_ms": round(ins_ms, 4), "query_ms": round(qry_ms, 4),
                    "insert_mops": round(n / ins_ms / 1e3, 1), "query_mops": round(nq / qry_ms / 1e3, 1),
                    "remove_mops": round(len(rem) / rem_ms / 1e3, 1),
                    "insert_failures": int((~okn).sum())},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clocks,
        "e2e": e2e,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args)
    if rank == 0:
        print(json.dumps(out))
    del table


def run_e2e(args, table, keys, vals, qkeys, dev, world):
    """The same step through the public API from pinned host buffers: the H2D
    copies of the step's keys / values / query keys and the D2H read of the
    query results and insert report are inside the timed region.  Copies are
    chunked and overlapped with the kernels: uploads on one stream, downloads
    on another (PCIe carries both directions at once), kernels on a third."""
    import torch

    n, nq = len(keys), len(qkeys)
    h_keys = torch.from_numpy(keys.view(np.int64)).pin_memory()
    h_vals = torch.from_numpy(vals.view(np.int64)).pin_memory()
    h_q = torch.from_numpy(qkeys.view(np.int64)).pin_memory()
    h_ok = torch.empty(n, dtype=torch.uint8).pin_memory()
    h_found = torch.empty(nq, dtype=torch.uint8).pin_memory()
    h_qv = torch.empty(nq, dtype=torch.int64).pin_memory()
    d_keys = torch.empty(n, dtype=torch.int64, device=dev)
    d_vals = torch.empty(n, dtype=torch.int64, device=dev)
    d_q = torch.empty(nq, dtype=torch.int64, device=dev)
    ok = torch.empty(n, dtype=torch.uint8, device=dev)
    found = torch.empty(nq, dtype=torch.uint8, device=dev)
    qv = torch.empty(nq, dtype=torch.int64, device=dev)
    h2d_s = torch.cuda.Stream(dev)  # host -> device copies
    d2h_s = torch.cuda.Stream(dev)  # device -> host copies (PCIe is full duplex: both directions at once)
    comp_s = torch.cuda.Stream(dev)
    chunks = 8

    def bounds(total):
        return [(total * i // chunks, total * (i + 1) // chunks) for i in range(chunks)]

    def step():
        table.clear(comp_s)
        for lo, hi in bounds(n):  # insert inputs chunk by chunk, each insert as soon as its chunk landed
            with torch.cuda.stream(h2d_s):
                d_keys[lo:hi].copy_(h_keys[lo:hi], non_blocking=True)
                d_vals[lo:hi].copy_(h_vals[lo:hi], non_blocking=True)
                e = torch.cuda.Event()
                e.record(h2d_s)
            comp_s.wait_event(e)
            table.bulk_insert(d_keys[lo:hi], d_vals[lo:hi], ok[lo:hi], None, comp_s)
        ins_done = torch.cuda.Event()
        ins_done.record(comp_s)
        d2h_s.wait_event(ins_done)
        with torch.cuda.stream(d2h_s):
            h_ok.copy_(ok, non_blocking=True)  # overlaps the query uploads
        for lo, hi in bounds(nq):
            with torch.cuda.stream(h2d_s):  # uploads overlap the inserts still running
                d_q[lo:hi].copy_(h_q[lo:hi], non_blocking=True)
                e = torch.cuda.Event()
                e.record(h2d_s)
            comp_s.wait_event(e)
            table.bulk_query(d_q[lo:hi], qv[lo:hi], found[lo:hi], None, comp_s)
            e = torch.cuda.Event()
            e.record(comp_s)
            d2h_s.wait_event(e)
            with torch.cuda.stream(d2h_s):
                h_qv[lo:hi].copy_(qv[lo:hi], non_blocking=True)
                h_found[lo:hi].copy_(found[lo:hi], non_blocking=True)

    steps = max(2, min(args.steps, 5))
    for _ in range(2):
        step()
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    el = allreduce_max(el * 1e3, world) / 1e3
    assert (h_found[: n // 2].numpy().astype(bool) == h_ok[: n // 2].numpy().astype(bool)).all()
    value = (n + nq) * steps * world / el / 1e6
    # the link itself: one large pinned copy each way, timed on the device
    probe = 1 << 30
    hb = torch.empty(probe, dtype=torch.uint8).pin_memory()
    db = torch.empty(probe, dtype=torch.uint8, device=dev)
    link = {}
    for name, dst, src in (("h2d", db, hb), ("d2h", hb, db)):
        for _ in range(2):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            dst.copy_(src, non_blocking=True)
            e1.record()
            torch.cuda.synchronize()
        link[name] = probe / (e0.elapsed_time(e1) / 1e3) / 1e9
    del hb, db
    h2d_rate = (16 * n + 8 * nq) * steps / el / 1e9
    return {"value": round(value, 1), "unit": "Mops/s", "h2d_bytes_per_step": 16 * n + 8 * nq,
            "d2h_bytes_per_step": n + 9 * nq, "steps": steps,
            "link_h2d_gbs": round(link["h2d"], 1), "link_d2h_gbs": round(link["d2h"], 1),
            "h2d_gbs_achieved": round(h2d_rate, 1), "h2d_frac_of_link": round(h2d_rate / link["h2d"], 3),
            "note": "host-timed around cudaMemcpyAsync H2D (pinned) + kernels + D2H, 8 chunks per phase, "
                    "uploads and downloads on separate streams"}


# ------------------------------------------------------------------ CPU legs
def cpu_baseline(args, threads: int | None = None):
    from oracle import pyoracle as po

    keys, vals, qkeys = make_inputs()
    cores = threads or po.online_cores()
    t = po.OracleTable(0, TILE, [(NSLOTS, BUCKET, PROBES, 0, 0)], SEED)
    t0 = time.perf_counter()
    t.insert_many(keys, vals, threads=cores)
    t.query_many(qkeys, threads=cores)
    el = time.perf_counter() - t0
    return {"value": round((len(keys) + len(qkeys)) / el / 1e6, 2), "unit": "Mops/s", "cores": cores,
            "kind": "port", "seconds": round(el, 2),
            "sample": "one full step (2^26-slot table, 60.4M inserts + 60.4M queries) on the multithreaded "
                      "host port of the reference's table semantics (oracle/poggers_oracle.c)"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    if args.ref_target == "cuda":
        return run_reference_cuda(args)
    from oracle import pyoracle as po

    keys, vals, qkeys = make_inputs()
    cores = po.online_cores()
    t = po.OracleTable(0, TILE, [(NSLOTS, BUCKET, PROBES, 0, 0)], SEED)
    n, nq = len(keys), len(qkeys)

    # a step is the whole workload, as on the GPU: clear the table, insert
    # every key, query every query key (about 2 s on 16 host cores)
    def step():
        t.clear()
        t.insert_many(keys, vals, threads=cores)
        t.query_many(qkeys, threads=cores)
        return n + nq

    for _ in range(args.warmup):
        step()
    ops = 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ops += step()
    el = time.perf_counter() - t0
    value = ops / el / 1e6
    sample = ("every step the whole workload (clear the 2^26-slot table, 60.4M inserts, 60.4M queries) on the "
              "multithreaded host port of the reference's table semantics (oracle/poggers_oracle.c); the "
              "reference has no CPU implementation")
    out = {"impl": "reference", "metric": METRIC, "value": round(value, 2), "unit": "Mops/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(el / args.steps * 1e3, 2),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
           "data": "synthetic (seeded splitmix64 keys)",
           "config": {"workload": WORKLOAD, "slots": NSLOTS, "inserts": len(keys), "queries": len(qkeys)},
           "cpu_baseline": {"value": round(value, 2), "unit": "Mops/s", "cores": cores, "kind": "port",
                            "sample": sample},
           "e2e": {"value": round(value, 2), "unit": "Mops/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def run_reference_cuda(args):
    """The reference's own CUDA build (oracle/_ref/libpoggers_refcuda.so) on this GPU:
    same table, same keys, reference kernel shape (one tile per key, 1024-thread blocks)."""
    import torch
    from oracle import pyrefcuda as rc

    if not rc.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libpoggers_refcuda.so not built"}))
        return
    dev = torch.device("cuda", torch.cuda.current_device())
    keys, vals, qkeys = make_inputs()
    n, nq = len(keys), len(qkeys)
    d_keys = torch.from_numpy(keys.view(np.int64)).to(dev)
    d_vals = torch.from_numpy(vals.view(np.int64)).to(dev)
    d_q = torch.from_numpy(qkeys.view(np.int64)).to(dev)
    ok = torch.empty(n, dtype=torch.uint8, device=dev)
    found = torch.empty(nq, dtype=torch.uint8, device=dev)
    qv = torch.empty(nq, dtype=torch.int64, device=dev)
    t = rc.RefTable(rc.KIND_HT_DOUBLE_B8, NSLOTS, 0, SEED)
    slots, nb = t.level(0)
    stream = torch.cuda.current_stream()
    import ctypes as C
    cudart = C.CDLL("libcudart.so.12")
    cudart.cudaMemsetAsync.argtypes = [C.c_void_p, C.c_int, C.c_size_t, C.c_void_p]

    def step(ev=None):
        cudart.cudaMemsetAsync(slots, 0, nb * BUCKET * 16, stream.cuda_stream)
        if ev:
            ev[0].record(stream)
        t.bulk(rc.OP_INSERT, d_keys, d_vals, ok, stream=stream)
        if ev:
            ev[1].record(stream)
        t.bulk(rc.OP_QUERY, d_q, None, found, qv, stream=stream)
        if ev:
            ev[2].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    sampler = ClockSampler(dev.index)
    sampler.start()
    time.sleep(0.3)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for k in range(args.steps):
        step(evs[k])
    t1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = t0.elapsed_time(t1)
    ins_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in evs)
    qry_ms = statistics.mean(e[1].elapsed_time(e[2]) for e in evs)
    value = (n + nq) * args.steps / (ms / 1e3) / 1e6
    print(json.dumps({"impl": "reference", "target": "cuda", "metric": METRIC, "value": round(value, 1),
                      "unit": "Mops/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                      "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True, "dtype": "u64",
                      "config": {"workload": WORKLOAD, "build": "reference headers, nvcc -O3 sm_100a, no -G"},
                      "kernels": {"insert_ms": round(ins_ms, 4), "query_ms": round(qry_ms, 4),
                                  "insert_mops": round(n / ins_ms / 1e3, 1),
                                  "query_mops": round(nq / qry_ms / 1e3, 1)},
                      "clocks": clocks}))
    t.close()


# ------------------------------------------------------------------ plumbing
def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allreduce_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--ref-target", choices=["cpu", "cuda"], default="cpu")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--layout", choices=["fingerprints", "interleaved", "split"], default=LAYOUT)
    ap.add_argument("--insert-order", choices=["region", "batch"], default="region",
                    help="region: inserts counting-sorted by table region (default); batch: in batch order")
    ap.add_argument("--slots-log2", type=int, default=26,
                    help="table size (default 26 = the benchmark workload; smaller only for profiling captures)")
    args = ap.parse_args()
    global NSLOTS, WORKLOAD
    if args.slots_log2 != 26:
        NSLOTS = 1 << args.slots_log2
        WORKLOAD = WORKLOAD.replace("2^26", f"2^{args.slots_log2}")
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference" and args.ref_target == "cpu":
        # host-only arm: rank 0 alone runs it, others exit without work
        run_reference(args, rank, world)
        return
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_ours(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
