"""One logical table hash-partitioned over the GPUs of a process group.

No counterpart in the reference, whose tables live on one GPU.  Each rank (one
process per GPU) holds one shard as an ordinary table sized for its share of
the slots.  A bulk call on any rank:

1. routes its batch by owner on the device (`pg_route_by_shard`: a counting
   sort into one run per shard, plus the permutation back to batch order);
2. exchanges the run lengths, then the runs, with all-to-all collectives
   (NCCL over NVLink / NVSwitch on GPUs, gloo on the host);
3. runs the bulk operation on the keys it received, on its own shard;
4. sends the results back with the reverse all-to-all and scatters them into
   batch order (`pg_scatter_by_perm`).

Every rank must call the same operations in the same order (they are
collectives).  Payloads travel as byte views, so 16-bit values need no
16-bit collective type.  The routing hash is MurmurHash64A with its own seed
(`pg_host_shard_of`), independent of the shards' bucket hashes.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import replace

import poggers_b200 as pg

ROUTE_SEED = 0x5EED_0F_5A4D  # default routing seed


def _dist():
    import torch.distributed as dist
    return dist


class CudaShardBackend:
    """The shard on this rank's GPU: a pg.Table plus the routing kernels."""

    def __init__(self, config: "pg.TableConfig", seed: int):
        self.table = pg.Table(config, seed)
        self.format = config.format
        self.val_bytes = pg.VAL_BYTES[config.format]

    @property
    def device(self):
        import torch
        return torch.device("cuda", torch.cuda.current_device())

    def route(self, keys, vals, nshards: int, route_seed: int):
        import torch
        n = keys.numel()
        sk = torch.empty(n, dtype=torch.int64, device=keys.device)
        sv = None if vals is None else torch.empty_like(vals)
        perm = torch.empty(n, dtype=torch.int32, device=keys.device)
        counts = torch.zeros(2 * nshards, dtype=torch.int64, device=keys.device)
        vb = 0 if vals is None else vals.element_size()
        st = pg.lib().pg_route_by_shard(pg._ptr(keys), pg._ptr(vals), vb, n, nshards, route_seed, pg._ptr(sk),
                                        pg._ptr(sv), pg._ptr(perm), pg._ptr(counts), pg._stream(None))
        pg._check(st, "pg_route_by_shard")
        return sk, sv, perm, counts[:nshards].clone()

    def unpermute(self, src, perm):
        import torch
        out = torch.empty_like(src)
        st = pg.lib().pg_scatter_by_perm(pg._ptr(src), pg._ptr(perm), src.numel(), src.element_size(),
                                         pg._ptr(out), pg._stream(None))
        pg._check(st, "pg_scatter_by_perm")
        return out

    def local(self, op: str, keys, vals):
        """The bulk operation on this shard; returns {name: tensor} of per-key results."""
        import torch
        n = keys.numel()
        flags = torch.zeros(n, dtype=torch.uint8, device=keys.device)
        if op == "insert":
            self.table.bulk_insert(keys, vals, flags)
            return {"ok": flags}
        if op == "remove":
            self.table.bulk_remove(keys, flags)
            return {"ok": flags}
        vdt = {8: torch.int64, 2: torch.int16, 1: torch.uint8, 0: torch.int16}[self.val_bytes]
        out = torch.zeros(n, dtype=vdt, device=keys.device)
        self.table.bulk_query(keys, out if self.val_bytes else None, flags)
        return {"found": flags, "vals": out}


class ShardedTable:
    """A table of config.levels' total slots split evenly over the group's ranks."""

    def __init__(self, config: "pg.TableConfig", seed: int, group=None, route_seed: int = ROUTE_SEED,
                 backend=None):
        dist = _dist()
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.route_seed = route_seed
        local = replace(config, levels=[replace(L, nslots=-(-L.nslots // self.world)) for L in config.levels])
        self.local_config = local
        self.backend = backend if backend is not None else CudaShardBackend(local, seed)

    # -------------------------------------------------------------- plumbing
    @staticmethod
    def _as_bytes(t):
        import torch
        if t.numel() == 0:
            return torch.empty(0, dtype=torch.uint8, device=t.device)
        return t.contiguous().view(torch.uint8)

    @staticmethod
    def _from_bytes(b, dtype):
        import torch
        if b.numel() == 0:
            return torch.empty(0, dtype=dtype, device=b.device)
        return b.view(dtype)

    def _a2a(self, send, send_counts, recv_counts, like):
        """all-to-all of the per-shard runs of `send` (any element type, moved as bytes)."""
        import torch
        dist = _dist()
        eb = send.element_size()
        out = torch.empty(sum(recv_counts) * eb, dtype=torch.uint8, device=like.device)
        if self.world == 1:
            out.copy_(self._as_bytes(send))
        else:
            dist.all_to_all_single(out, self._as_bytes(send), [c * eb for c in recv_counts],
                                   [c * eb for c in send_counts], group=self.group)
        return self._from_bytes(out, send.dtype)

    def _counts(self, counts):
        import torch
        dist = _dist()
        if self.world == 1:
            return counts.tolist(), counts.tolist()
        recv = torch.empty_like(counts)
        dist.all_to_all_single(recv, counts, group=self.group)
        return counts.tolist(), recv.tolist()

    def _run(self, op: str, keys, vals=None):
        sk, sv, perm, counts = self.backend.route(keys, vals, self.world, self.route_seed)
        send, recv = self._counts(counts)
        rk = self._a2a(sk, send, recv, keys)
        rv = None if vals is None else self._a2a(sv, send, recv, vals)
        res = self.backend.local(op, rk, rv)
        out = {}
        for name, r in res.items():
            out[name] = self.backend.unpermute(self._a2a(r, recv, send, r), perm)
        return out

    # -------------------------------------------------------------- operations
    def insert(self, keys, vals=None):
        """ok flags per key of this rank's batch (collective)."""
        return self._run("insert", keys, vals)["ok"]

    def query(self, keys):
        """(found flags, values) per key of this rank's batch (collective)."""
        r = self._run("query", keys)
        return r["found"], r["vals"]

    def remove(self, keys):
        """removed flags per key of this rank's batch (collective)."""
        return self._run("remove", keys)["ok"]


def shard_of(key: int, nshards: int, route_seed: int = ROUTE_SEED) -> int:
    """Owner shard of a key (host)."""
    return pg.lib().pg_host_shard_of(C.c_uint64(key), C.c_uint64(route_seed), nshards)
