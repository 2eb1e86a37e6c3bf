"""Seeded synthetic workloads (keys, values, query mixes) for tests and the bench.

Keys come from splitmix64 (Steele, Lea & Flood 2014) over a counter: key i of
stream `seed` is mix(seed + (i + 1) * 0x9E3779B97F4A7C15).  The mix is a
bijection, so one stream never repeats a key.  The reference's test drivers
draw keys from OpenSSL RAND_bytes, unseeded (tests/src/test_mhm_tcf.cu:235-262);
a seeded stream with the same distribution (uniform 64-bit) replaces it so
every run is reproducible.
"""
from __future__ import annotations

import numpy as np

GAMMA = np.uint64(0x9E3779B97F4A7C15)
M1 = np.uint64(0xBF58476D1CE4E5B9)
M2 = np.uint64(0x94D049BB133111EB)
SENTINELS = (0, (1 << 64) - 1)  # empty and tombstone keys of key_val_pair<uint64,...>


def splitmix64(seed: int, n: int, start: int = 0) -> np.ndarray:
    i = np.arange(start + 1, start + n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + i * GAMMA
        z = (z ^ (z >> np.uint64(30))) * M1
        z = (z ^ (z >> np.uint64(27))) * M2
    return z ^ (z >> np.uint64(31))


def keys_without_sentinels(seed: int, n: int) -> np.ndarray:
    """n distinct keys with the table sentinels (0 and ~0) dropped."""
    k = splitmix64(seed, n)
    bad = (k == np.uint64(0)) | (k == np.uint64(SENTINELS[1]))
    if bad.any():
        extra = splitmix64(seed, int(bad.sum()), start=n)
        k = np.concatenate([k[~bad], extra])
    return k


def values_for(keys: np.ndarray, fmt_val_bytes: int, seed: int = 7) -> np.ndarray:
    """Deterministic values: a second splitmix stream, cut to the value width."""
    v = splitmix64(seed, len(keys))
    if fmt_val_bytes == 2:
        return (v & np.uint64(0xFFFF)).astype(np.uint16)
    return v


def fisher_yates_half(n: int, seed: int) -> np.ndarray:
    """Indices of a seeded random half of range(n) (the remove set of the HT workload)."""
    rng = np.random.default_rng(seed)
    return np.sort(rng.permutation(n)[: n // 2])


def _s64(x: int) -> int:
    return x - (1 << 64) if x >= (1 << 63) else x


def device_splitmix64(seed: int, n: int, start: int = 0, device="cuda"):
    """splitmix64(seed, n, start) computed by torch on `device` (int64 tensor with
    the same bits as the numpy stream), for workloads too large to build on the host."""
    import torch

    def lsr(x, s):
        return torch.bitwise_right_shift(x, s) & ((1 << (64 - s)) - 1)

    z = torch.arange(start + 1, start + n + 1, dtype=torch.int64, device=device)
    z = z * _s64(int(GAMMA)) + _s64(seed % (1 << 64))
    z = (z ^ lsr(z, 30)) * _s64(int(M1))
    z = (z ^ lsr(z, 27)) * _s64(int(M2))
    z = z ^ lsr(z, 31)
    # the table sentinels 0 and ~0 become 1 and ~0 - 1 (a 2^-63 event per key)
    z = torch.where(z == 0, torch.ones_like(z), z)
    return torch.where(z == -1, torch.full_like(z, -2), z)


def device_zipf_ranks(n_items: int, count: int, a: float, seed: int, device="cuda"):
    """`count` ranks in [0, n_items) drawn from a bounded power law with exponent a
    (Zipf(a), by inverting the continuous CDF), on `device` (int64)."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    u = torch.rand(count, dtype=torch.float64, device=device, generator=g)
    e = 1.0 - a
    x = (1.0 + u * ((n_items + 1.0) ** e - 1.0)) ** (1.0 / e)
    return (x.floor().to(torch.int64) - 1).clamp_(0, n_items - 1)
