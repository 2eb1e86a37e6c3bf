"""Helpers for the GPU tests: numpy <-> torch CUDA tensors and table drivers."""
from __future__ import annotations

import numpy as np


def to_dev(a: np.ndarray):
    import torch
    if a.dtype == np.uint64:
        return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()
    if a.dtype == np.uint16:
        return torch.from_numpy(np.ascontiguousarray(a).view(np.int16)).cuda()
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def val_dtype(fmt: int):
    import torch
    return torch.int64 if fmt == 0 else torch.int16


def vals_np(fmt: int, vals_u64: np.ndarray) -> np.ndarray:
    return vals_u64.astype(np.uint64) if fmt == 0 else (vals_u64 & np.uint64(0xFFFF)).astype(np.uint16)


def u64(t) -> np.ndarray:
    a = t.cpu().numpy()
    if a.dtype == np.int16:
        return a.view(np.uint16).astype(np.uint64)
    return a.view(np.uint64) if a.dtype == np.int64 else a.astype(np.uint64)


class Driver:
    """Runs insert / query / remove on a product table with numpy inputs."""

    def __init__(self, table):
        self.t = table
        self.fmt = table.format

    def insert(self, keys, vals_u64=None):
        import torch
        k = to_dev(keys)
        v = None if vals_u64 is None or self.fmt == 2 else to_dev(vals_np(self.fmt, vals_u64))
        ok = torch.zeros(len(keys), dtype=torch.uint8, device="cuda")
        fails = torch.zeros(1, dtype=torch.int64, device="cuda")
        self.t.bulk_insert(k, v, ok, fails)
        torch.cuda.synchronize()
        okn = ok.cpu().numpy().astype(bool)
        assert int(fails.item()) == int((~okn).sum())
        return okn

    def query(self, keys):
        import torch
        k = to_dev(keys)
        f = torch.zeros(len(keys), dtype=torch.uint8, device="cuda")
        v = torch.full((len(keys),), -1, dtype=val_dtype(self.fmt), device="cuda")
        hits = torch.zeros(1, dtype=torch.int64, device="cuda")
        self.t.bulk_query(k, v, f, hits)
        torch.cuda.synchronize()
        fn = f.cpu().numpy().astype(bool)
        assert int(hits.item()) == int(fn.sum())
        return fn, u64(v)

    def remove(self, keys):
        import torch
        k = to_dev(keys)
        ok = torch.zeros(len(keys), dtype=torch.uint8, device="cuda")
        hits = torch.zeros(1, dtype=torch.int64, device="cuda")
        self.t.bulk_remove(k, ok, hits)
        torch.cuda.synchronize()
        okn = ok.cpu().numpy().astype(bool)
        assert int(hits.item()) == int(okn.sum())
        return okn
