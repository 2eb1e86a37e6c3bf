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
