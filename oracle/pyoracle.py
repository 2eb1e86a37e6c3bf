"""ctypes loader for the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this.
It wraps oracle/_build/libpoggers_oracle.so (the C restatement of the
reference's table algorithms) and, when present, oracle/_ref/*.so (the
reference's own code compiled from its sources by oracle/Makefile).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libpoggers_oracle.so"
REFHOST_PATH = HERE / "_ref" / "libpoggers_refhost.so"
REFCUDA_PATH = HERE / "_ref" / "libpoggers_refcuda.so"

FMT_KV64, FMT_TAGVAL16, FMT_TAG16 = 0, 1, 2
SCHEME_BUCKET, SCHEME_TWO_CHOICE, SCHEME_TWO_CHOICE_BUCKETED, SCHEME_LINEAR_BUCKETED = 0, 1, 2, 3
BOP_INSERT, BOP_QUERY, BOP_REMOVE, BOP_INSERT_DELETE, BOP_INSERT_IF_NOT_EXISTS, BOP_INSERT_IF_NOT_EXISTS_DELETE = range(6)
PROBE_DOUBLE, PROBE_LINEAR, PROBE_P2, PROBE_XOR_P2 = 0, 1, 2, 3
SLOT_BYTES = {FMT_KV64: 16, FMT_TAGVAL16: 4, FMT_TAG16: 2}


class LevelCfg(C.Structure):
    _fields_ = [("nslots", C.c_uint64), ("bucket_size", C.c_uint32), ("max_probes", C.c_uint32),
                ("scheme", C.c_uint32), ("probe", C.c_uint32)]


class BCfg(C.Structure):
    _fields_ = [("tag_bits", C.c_uint32), ("nlevels", C.c_uint32), ("pad0", C.c_uint32), ("pad1", C.c_uint32),
                ("lv", LevelCfg * 2)]


class Cfg(C.Structure):
    _fields_ = [("format", C.c_uint32), ("partition", C.c_uint32), ("nlevels", C.c_uint32),
                ("pad", C.c_uint32), ("lv", LevelCfg * 2)]


_lib = None
_refhost = None

U64P = C.POINTER(C.c_uint64)
U8P = C.POINTER(C.c_uint8)


def build() -> None:
    """Compile the C restatement (and the reference host pin when the reference is present)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        L.pgo_murmur64a.restype = C.c_uint64
        L.pgo_murmur64a.argtypes = [C.c_void_p, C.c_int, C.c_uint64]
        L.pgo_tag16.restype = C.c_uint64
        L.pgo_tag16.argtypes = [C.c_uint64]
        L.pgo_probe_values.restype = C.c_int
        L.pgo_probe_values.argtypes = [C.c_uint32, C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint32, U64P]
        L.pgo_table_create.restype = C.c_void_p
        L.pgo_table_create.argtypes = [C.POINTER(Cfg), C.c_uint64]
        L.pgo_table_destroy.argtypes = [C.c_void_p]
        L.pgo_table_clear.argtypes = [C.c_void_p]
        for f in ("pgo_level_nbuckets", "pgo_level_bytes", "pgo_level_seed"):
            getattr(L, f).restype = C.c_uint64
            getattr(L, f).argtypes = [C.c_void_p, C.c_int]
        L.pgo_level_data.restype = C.c_void_p
        L.pgo_level_data.argtypes = [C.c_void_p, C.c_int]
        L.pgo_insert.restype = C.c_int
        L.pgo_insert.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64]
        L.pgo_query.restype = C.c_int
        L.pgo_query.argtypes = [C.c_void_p, C.c_uint64, U64P]
        L.pgo_remove.restype = C.c_int
        L.pgo_remove.argtypes = [C.c_void_p, C.c_uint64]
        L.pgo_bulk_insert.restype = C.c_uint64
        L.pgo_bulk_insert.argtypes = [C.c_void_p, U64P, U64P, C.c_uint64, U8P]
        L.pgo_bulk_query.restype = C.c_uint64
        L.pgo_bulk_query.argtypes = [C.c_void_p, U64P, C.c_uint64, U64P, U8P]
        L.pgo_bulk_remove.restype = C.c_uint64
        L.pgo_bulk_remove.argtypes = [C.c_void_p, U64P, C.c_uint64, U8P]
        L.pgo_count_fill.restype = C.c_uint64
        L.pgo_count_fill.argtypes = [C.c_void_p, C.c_int]
        L.pgo_mt_bulk_insert.restype = C.c_uint64
        L.pgo_mt_bulk_insert.argtypes = [C.c_void_p, U64P, U64P, C.c_uint64, U8P, C.c_int]
        L.pgo_mt_bulk_query.restype = C.c_uint64
        L.pgo_mt_bulk_query.argtypes = [C.c_void_p, U64P, C.c_uint64, U64P, U8P, C.c_int]
        L.pgo_mt_bulk_remove.restype = C.c_uint64
        L.pgo_mt_bulk_remove.argtypes = [C.c_void_p, U64P, C.c_uint64, U8P, C.c_int]
        L.pgo_online_cores.restype = C.c_int
        L.pgo_splitmix64_fill.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, U64P]
        L.pgo_slab_create.restype = C.c_void_p
        L.pgo_slab_create.argtypes = [C.c_uint64]
        L.pgo_slab_destroy.argtypes = [C.c_void_p]
        for f in ("pgo_slab_capacity", "pgo_slab_free_objects"):
            getattr(L, f).restype = C.c_uint64
            getattr(L, f).argtypes = [C.c_void_p]
        L.pgo_slab_malloc.restype = C.c_uint64
        L.pgo_slab_malloc.argtypes = [C.c_void_p, C.c_uint64, U64P]
        L.pgo_slab_free.restype = C.c_uint64
        L.pgo_slab_free.argtypes = [C.c_void_p, C.c_uint64, U64P]
        L.pgo_btag.restype = C.c_uint64
        L.pgo_btag.argtypes = [C.c_uint32, C.c_uint64]
        L.pgo_btable_create.restype = C.c_void_p
        L.pgo_btable_create.argtypes = [C.POINTER(BCfg), C.c_uint64]
        L.pgo_btable_destroy.argtypes = [C.c_void_p]
        for f in ("pgo_btable_level_bytes", "pgo_btable_level_nbuckets"):
            getattr(L, f).restype = C.c_uint64
            getattr(L, f).argtypes = [C.c_void_p, C.c_int]
        L.pgo_btable_level_data.restype = C.c_void_p
        L.pgo_btable_level_data.argtypes = [C.c_void_p, C.c_int]
        L.pgo_btable_op.restype = C.c_int
        L.pgo_btable_op.argtypes = [C.c_void_p, C.c_int, C.c_uint64, C.c_uint64, U64P, C.POINTER(C.c_int)]
        L.pgo_btable_bulk.restype = C.c_uint64
        L.pgo_btable_bulk.argtypes = [C.c_void_p, C.c_int, U64P, U64P, C.c_uint64, U64P, U8P, U8P]
        L.pgo_btable_count_fill.restype = C.c_uint64
        L.pgo_btable_count_fill.argtypes = [C.c_void_p, C.c_int]
        L.pgo_rslab_create.restype = C.c_void_p
        L.pgo_rslab_create.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_uint64]
        L.pgo_rslab_destroy.argtypes = [C.c_void_p]
        for f in ("pgo_rslab_report_fill", "pgo_rslab_report_max", "pgo_rslab_short_pins", "pgo_rslab_lost_words"):
            getattr(L, f).restype = C.c_uint64
            getattr(L, f).argtypes = [C.c_void_p]
        L.pgo_rslab_malloc.restype = C.c_uint64
        L.pgo_rslab_malloc.argtypes = [C.c_void_p, C.c_int, C.c_int, U64P]
        L.pgo_rslab_free.restype = C.c_int
        L.pgo_rslab_free.argtypes = [C.c_void_p, C.c_uint64]
        _lib = L
    return _lib


def refhost():
    """The reference's own hash / probe code compiled for the host, or None."""
    global _refhost
    if _refhost is None and REFHOST_PATH.exists():
        L = C.CDLL(str(REFHOST_PATH))
        L.refh_murmur64a.restype = C.c_uint64
        L.refh_murmur64a.argtypes = [C.c_uint64, C.c_uint64]
        L.refh_probe_values.restype = C.c_int
        L.refh_probe_values.argtypes = [C.c_int, C.c_uint64, C.c_uint64, C.c_uint64, U64P, C.c_int]
        _refhost = L
    return _refhost


def _p64(a):
    return None if a is None else a.ctypes.data_as(U64P)


def _p8(a):
    return None if a is None else a.ctypes.data_as(U8P)


def splitmix64(seed: int, n: int, start: int = 0) -> np.ndarray:
    out = np.empty(n, dtype=np.uint64)
    lib().pgo_splitmix64_fill(seed, start, n, _p64(out))
    return out


def murmur64a(key: int, seed: int) -> int:
    k = C.c_uint64(key)
    return lib().pgo_murmur64a(C.byref(k), 8, seed)


def probe_values(probe: int, seed: int, fmt: int, key: int, max_probes: int) -> list[int]:
    out = np.zeros(max(max_probes, 1), dtype=np.uint64)
    n = lib().pgo_probe_values(probe, seed, fmt, key, max_probes, _p64(out))
    return [int(x) for x in out[:n]]


def make_cfg(fmt: int, partition: int, levels: list[tuple]) -> Cfg:
    """levels: [(nslots, bucket_size, max_probes, scheme, probe), ...]"""
    c = Cfg()
    c.format, c.partition, c.nlevels = fmt, partition, len(levels)
    for i, lv in enumerate(levels):
        c.lv[i] = LevelCfg(*lv)
    return c


class OracleTable:
    """Sequential model of one reference table (static_table semantics)."""

    def __init__(self, fmt: int, partition: int, levels: list[tuple], seed: int):
        self.cfg = make_cfg(fmt, partition, levels)
        self.fmt = fmt
        self.h = lib().pgo_table_create(C.byref(self.cfg), seed)
        if not self.h:
            raise ValueError("invalid oracle table configuration")

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().pgo_table_destroy(h)
            self.h = None

    @property
    def nlevels(self) -> int:
        return self.cfg.nlevels

    def clear(self):
        lib().pgo_table_clear(self.h)

    def nbuckets(self, level: int) -> int:
        return lib().pgo_level_nbuckets(self.h, level)

    def level_bytes(self, level: int) -> bytes:
        n = lib().pgo_level_bytes(self.h, level)
        return C.string_at(lib().pgo_level_data(self.h, level), n)

    def insert_many(self, keys, vals=None, threads: int | None = None):
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        vals = None if vals is None else np.ascontiguousarray(vals, dtype=np.uint64)
        ok = np.zeros(len(keys), dtype=np.uint8)
        if threads is None:
            lib().pgo_bulk_insert(self.h, _p64(keys), _p64(vals), len(keys), _p8(ok))
        else:
            lib().pgo_mt_bulk_insert(self.h, _p64(keys), _p64(vals), len(keys), _p8(ok), threads)
        return ok.astype(bool)

    def query_many(self, keys, threads: int | None = None):
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        vals = np.zeros(len(keys), dtype=np.uint64)
        found = np.zeros(len(keys), dtype=np.uint8)
        if threads is None:
            lib().pgo_bulk_query(self.h, _p64(keys), len(keys), _p64(vals), _p8(found))
        else:
            lib().pgo_mt_bulk_query(self.h, _p64(keys), len(keys), _p64(vals), _p8(found), threads)
        return found.astype(bool), vals

    def remove_many(self, keys, threads: int | None = None):
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        ok = np.zeros(len(keys), dtype=np.uint8)
        if threads is None:
            lib().pgo_bulk_remove(self.h, _p64(keys), len(keys), _p8(ok))
        else:
            lib().pgo_mt_bulk_remove(self.h, _p64(keys), len(keys), _p8(ok), threads)
        return ok.astype(bool)

    def count_fill(self, level: int) -> int:
        return lib().pgo_count_fill(self.h, level)


def online_cores() -> int:
    return lib().pgo_online_cores()


class OracleSlab:
    """Sequential model of one fixed-size object pool (counts only)."""

    def __init__(self, num_allocs: int):
        self.h = lib().pgo_slab_create(num_allocs)

    def __del__(self):
        if getattr(self, "h", None):
            lib().pgo_slab_destroy(self.h)
            self.h = None

    @property
    def capacity(self) -> int:
        return lib().pgo_slab_capacity(self.h)

    @property
    def free_objects(self) -> int:
        return lib().pgo_slab_free_objects(self.h)

    def malloc(self, n: int):
        out = np.zeros(n, dtype=np.uint64)
        fails = lib().pgo_slab_malloc(self.h, n, _p64(out))
        return out, fails

    def free(self, offsets) -> int:
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        return lib().pgo_slab_free(self.h, len(offsets), _p64(offsets))


class OracleBucketed:
    """Sequential model of the reference's bucketed_table with packed slots
    (del_TCF: tag_bits 16; del_TCF_small: tag_bits 8).
    levels: [(nslots, bucket_size, max_probes, scheme, probe), ...]"""

    def __init__(self, tag_bits: int, levels: list[tuple], seed: int):
        c = BCfg()
        c.tag_bits, c.nlevels = tag_bits, len(levels)
        for i, lv in enumerate(levels):
            c.lv[i] = LevelCfg(*lv)
        self.cfg = c
        self.h = lib().pgo_btable_create(C.byref(c), seed)
        if not self.h:
            raise ValueError("invalid bucketed oracle configuration")

    def __del__(self):
        if getattr(self, "h", None):
            lib().pgo_btable_destroy(self.h)
            self.h = None

    def level_bytes(self, level: int) -> bytes:
        n = lib().pgo_btable_level_bytes(self.h, level)
        return C.string_at(lib().pgo_btable_level_data(self.h, level), n)

    def nbuckets(self, level: int) -> int:
        return lib().pgo_btable_level_nbuckets(self.h, level)

    def bulk(self, op: int, keys, vals=None):
        """(ok, out values, found) after running `op` on every key in batch order."""
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        vals = None if vals is None else np.ascontiguousarray(vals, dtype=np.uint64)
        out = np.zeros(len(keys), dtype=np.uint64)
        ok = np.zeros(len(keys), dtype=np.uint8)
        found = np.zeros(len(keys), dtype=np.uint8)
        lib().pgo_btable_bulk(self.h, op, _p64(keys), _p64(vals), len(keys), _p64(out), _p8(ok), _p8(found))
        return ok.astype(bool), out, found.astype(bool)

    def count_fill(self, level: int) -> int:
        return lib().pgo_btable_count_fill(self.h, level)


RSLAB_REFUSED, RSLAB_FREED, RSLAB_RETURNED, RSLAB_EMPTIED_PINNED = range(4)


class RefSlab:
    """Sequential restatement of the reference's one_size_slab_allocator<E>
    (per-SM pinned slabs, whole-word claims with a per-SM cache, pivot, pool)."""

    def __init__(self, num_allocs: int, sms: int, extra_blocks: int, seed: int = 1):
        self.h = lib().pgo_rslab_create(num_allocs, sms, extra_blocks, seed)
        if not self.h:
            raise ValueError("invalid slab configuration")

    def __del__(self):
        if getattr(self, "h", None):
            lib().pgo_rslab_destroy(self.h)
            self.h = None

    def report_fill(self) -> int:
        return lib().pgo_rslab_report_fill(self.h)

    def report_max(self) -> int:
        return lib().pgo_rslab_report_max(self.h)

    @property
    def short_pins(self) -> int:
        return lib().pgo_rslab_short_pins(self.h)

    @property
    def lost_words(self) -> int:
        return lib().pgo_rslab_lost_words(self.h)

    def malloc(self, sm: int, group: int):
        """One malloc() by `group` lanes of a warp on SM `sm`: (offsets or ~0, NULL count)."""
        out = np.zeros(32, dtype=np.uint64)
        nulls = lib().pgo_rslab_malloc(self.h, sm, group, _p64(out))
        return out[:group], int(nulls)

    def free(self, offset: int) -> int:
        return lib().pgo_rslab_free(self.h, int(offset))
