"""CPU tests of the multi-GPU sharded table's host logic: routing, the
all-to-all exchange protocol and the return of results to batch order, run
as world_size-2 gloo process groups on the host.  The shards are the oracle's
tables and the routing is the host owner function, so what is exercised is
everything above the device kernels (the kernels themselves are tested on a
GPU in tests/test_sharded_gpu.py)."""
from __future__ import annotations

import os
import socket
from datetime import timedelta

import numpy as np
import pytest

from poggers_b200 import workload as wl

ROUTE_SEED = 0x5EED_0F_5A4D


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def host_owner(keys: np.ndarray, nshards: int, seed: int = ROUTE_SEED) -> np.ndarray:
    import poggers_b200 as pg
    f = pg.lib().pg_host_shard_of
    return np.array([f(int(k), seed, nshards) for k in keys], dtype=np.int64)


class HostShardBackend:
    """Oracle table as the shard, numpy routing: the same interface as
    poggers_b200.sharded.CudaShardBackend, on CPU tensors."""

    def __init__(self, levels, seed):
        from oracle import pyoracle
        self.t = pyoracle.OracleTable(0, 4, levels, seed)

    def route(self, keys, vals, nshards, route_seed):
        import torch
        k = keys.numpy().view(np.uint64)
        owner = host_owner(k, nshards, route_seed)
        perm = np.argsort(owner, kind="stable")
        counts = np.bincount(owner, minlength=nshards).astype(np.int64)
        sk = torch.from_numpy(k[perm].view(np.int64).copy())
        sv = None if vals is None else vals[torch.from_numpy(perm)]
        return sk, sv, torch.from_numpy(perm.astype(np.int32)), torch.from_numpy(counts)

    def unpermute(self, src, perm):
        out = src.clone()
        out[perm.long()] = src
        return out

    def local(self, op, keys, vals):
        import torch
        k = keys.numpy().view(np.uint64)
        if op == "insert":
            v = None if vals is None else vals.numpy().view(np.uint64)
            ok = self.t.insert_many(k, v)
            return {"ok": torch.from_numpy(ok.astype(np.uint8))}
        if op == "remove":
            return {"ok": torch.from_numpy(self.t.remove_many(k).astype(np.uint8))}
        f, v = self.t.query_many(k)
        return {"found": torch.from_numpy(f.astype(np.uint8)), "vals": torch.from_numpy(v.view(np.int64).copy())}


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
        import poggers_b200 as pg
        from poggers_b200.sharded import ShardedTable
        cfg = pg.data_structs.hash_table_64(1 << 14, bucket=8)
        st = ShardedTable(cfg, 43, backend=HostShardBackend([((1 << 14) // world, 8, 20, 0, 0)], 43))
        assert st.local_config.levels[0].nslots == (1 << 14) // world
        # every rank inserts its own batch
        mine = wl.keys_without_sentinels(100 + rank, 3000)
        vals = wl.values_for(mine, 8, 7 + rank)
        ok = st.insert(torch.from_numpy(mine.view(np.int64)), torch.from_numpy(vals.view(np.int64)))
        assert ok.numpy().all(), "insert failures in a half-full table"
        # this rank's shard holds exactly the keys of every rank that route to it
        allk = np.concatenate([wl.keys_without_sentinels(100 + r, 3000) for r in range(world)])
        allv = np.concatenate([wl.values_for(wl.keys_without_sentinels(100 + r, 3000), 8, 7 + r)
                               for r in range(world)])
        owner = host_owner(allk, world)
        assert st.backend.t.count_fill(0) == int((owner == rank).sum())
        # every rank queries every rank's keys plus absent ones, in its own order
        rng = np.random.default_rng(rank)
        absent = wl.keys_without_sentinels(900 + rank, 1000)
        qk = np.concatenate([allk, absent])
        order = rng.permutation(len(qk))
        f, v = st.query(torch.from_numpy(qk[order].view(np.int64)))
        f = f.numpy().astype(bool)
        v = v.numpy().view(np.uint64)
        exp_f = np.concatenate([np.ones(len(allk), bool), np.zeros(len(absent), bool)])[order]
        exp_v = np.concatenate([allv, np.zeros(len(absent), np.uint64)])[order]
        assert (f == exp_f).all() and (v == exp_v).all()
        # rank 0 removes a third of rank 1's keys; every rank sees it
        rem = wl.keys_without_sentinels(100 + (1 % world), 3000)[:1000] if rank == 0 else np.zeros(0, np.uint64)
        r = st.remove(torch.from_numpy(rem.view(np.int64)))
        assert r.numpy().all()
        f2, _ = st.query(torch.from_numpy(allk.view(np.int64)))
        gone = np.isin(allk, wl.keys_without_sentinels(100 + (1 % world), 3000)[:1000])
        assert (f2.numpy().astype(bool) == ~gone).all()
        # an empty batch on one rank still takes part in the collectives
        e = torch.zeros(0, dtype=torch.int64) if rank == 1 else torch.from_numpy(allk[:10].view(np.int64))
        f3, _ = st.query(e)
        assert len(f3) == len(e)
        dist.barrier()
        q.put((rank, "ok"))
    except Exception as ex:  # reported to the parent
        import traceback
        q.put((rank, f"{type(ex).__name__}: {ex}\n{traceback.format_exc()}"))
    finally:
        if dist.is_initialized():
            dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_sharded_table_over_gloo(world):
    import torch.multiprocessing as mp
    import queue
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = {}
    for _ in range(world):
        try:
            r, msg = q.get(timeout=180)
        except queue.Empty:
            break
        results[r] = msg
    for p in procs:
        p.join(timeout=120)
        if p.is_alive():
            p.kill()
    assert all(results.get(r) == "ok" for r in range(world)), results


def test_owner_function_is_uniform_and_matches_host_helper():
    import poggers_b200 as pg
    keys = wl.keys_without_sentinels(5, 20000)
    for n in (1, 2, 3, 8):
        o = host_owner(keys, n)
        assert o.min() >= 0 and o.max() < n
        counts = np.bincount(o, minlength=n)
        assert counts.min() > 0.9 * len(keys) / n
    # the multiply-shift owner: high bits of murmur(key, seed) * n
    k = int(keys[0])
    h = pg.lib().pg_host_murmur64a(k, ROUTE_SEED)
    assert pg.lib().pg_host_shard_of(k, ROUTE_SEED, 8) == (h * 8) >> 64


def _bench_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
        import bench
        bench.barrier(world)
        m = bench.allreduce_max(10.0 + rank, world)
        q.put((rank, "ok" if m == 10.0 + world - 1 else f"max {m}"))
    except Exception as ex:
        q.put((rank, f"{type(ex).__name__}: {ex}"))
    finally:
        if dist.is_initialized():
            dist.destroy_process_group()


def test_bench_rank_timing_helpers_over_gloo():
    """bench.py's multi-rank timing takes the max over ranks of the device time."""
    import queue
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_bench_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = {}
    for _ in range(2):
        try:
            r, msg = q.get(timeout=120)
        except queue.Empty:
            break
        results[r] = msg
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert results == {0: "ok", 1: "ok"}, results
