"""poggers_b200 -- B200-native (sm_100a) POGGERS hot path.

Python host API over the C ABI of libpoggers_b200.so (include/poggers_b200.h).
Names follow the reference's template API so a reference user recognises
them:

    reference (C++ templates)                       here
    poggers::tables::static_table<...>              Table(TableConfig, seed)
    Table::generate_on_device(&sizing, seed)        Table.generate_on_device(config, sizing, seed)
    Table::free_on_device(table)                    table.free_on_device()
    insert / query / remove(tile, key[, val])       bulk_insert / bulk_query / bulk_remove
    poggers::data_structs::tcf                      data_structs.tcf(...)
    poggers::data_structs::hash_table_64            data_structs.hash_table_64(...)
    poggers::sizing::size_in_num_slots<N>(...)      sizing.size_in_num_slots(...)

Device buffers are torch CUDA tensors (or raw device addresses as ints).
The library must be built (poggers_b200/build.py); nothing here falls back
to a CPU path: a missing or unloadable library raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from pathlib import Path

_PKG = Path(__file__).resolve().parent
# POGGERS_B200_LIB selects another build of the same library (e.g. a variant
# compiled with different launch bounds, for a side-by-side measurement)
LIB_PATH = Path(os.environ.get("POGGERS_B200_LIB", str(_PKG / "libpoggers_b200.so")))

# ---- enums (include/poggers_b200.h)
PG_OK, PG_ERR_INVALID, PG_ERR_CUDA, PG_ERR_NOMEM, PG_ERR_UNSUPPORTED, PG_ERR_FULL, PG_ERR_TIMEOUT, PG_ERR_TOO_LARGE = range(8)
PG_STATIC_MAX_TABLES = 256
PG_STATIC_MAX_OPS = 8192
PG_DIAG_READ32, PG_DIAG_READ64, PG_DIAG_READ32_CAS, PG_DIAG_RED32, PG_DIAG_READ32_CAS_NEXT = 0, 1, 2, 3, 4
PG_TABLE_SPLIT_BUCKETS = 1
PG_TABLE_FINGERPRINTS = 2
FMT_KV64, FMT_TAGVAL16, FMT_TAG16, FMT_PACKED_TAGVAL16, FMT_PACKED_TAGVAL8 = 0, 1, 2, 3, 4
SCHEME_BUCKET, SCHEME_TWO_CHOICE, SCHEME_TWO_CHOICE_BUCKETED, SCHEME_LINEAR_BUCKETED = 0, 1, 2, 3
PROBE_DOUBLE, PROBE_LINEAR, PROBE_P2, PROBE_XOR_P2 = 0, 1, 2, 3
KEY_BYTES = {FMT_KV64: 8, FMT_TAGVAL16: 2, FMT_TAG16: 2, FMT_PACKED_TAGVAL16: 2, FMT_PACKED_TAGVAL8: 1}
VAL_BYTES = {FMT_KV64: 8, FMT_TAGVAL16: 2, FMT_TAG16: 0, FMT_PACKED_TAGVAL16: 2, FMT_PACKED_TAGVAL8: 1}
PACKED_FORMATS = (FMT_PACKED_TAGVAL16, FMT_PACKED_TAGVAL8)
SLOT_BYTES = {f: KEY_BYTES[f] + VAL_BYTES[f] for f in KEY_BYTES}


class PoggersError(RuntimeError):
    def __init__(self, status: int, what: str):
        self.status = status
        super().__init__(f"{what}: {status_string(status)} ({status})")


class _LevelConfig(C.Structure):
    _fields_ = [("nslots", C.c_uint64), ("bucket_size", C.c_uint32), ("max_probes", C.c_uint32),
                ("scheme", C.c_uint32), ("probe", C.c_uint32)]


class _TableConfig(C.Structure):
    _fields_ = [("format", C.c_uint32), ("tile", C.c_uint32), ("nlevels", C.c_uint32),
                ("flags", C.c_uint32), ("levels", _LevelConfig * 2)]


class _LevelInfo(C.Structure):
    _fields_ = [("nbuckets", C.c_uint64), ("nslots", C.c_uint64), ("bytes", C.c_uint64),
                ("seed", C.c_uint64), ("d_buckets", C.c_void_p)]


class _ServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("max_wave_keys", C.c_uint64),
                ("max_wave_requests", C.c_uint32), ("reserved", C.c_uint32)]


class _ServerTiming(C.Structure):
    _fields_ = [("waves", C.c_uint64), ("requests", C.c_uint64), ("keys", C.c_uint64),
                ("plan_s", C.c_double), ("copy_in_s", C.c_double), ("issue_s", C.c_double),
                ("copy_out_s", C.c_double), ("wait_busy_s", C.c_double), ("wait_idle_s", C.c_double)]


class _SlabInfo(C.Structure):
    _fields_ = [("pool", C.c_void_p), ("pool_bytes", C.c_uint64), ("object_bytes", C.c_uint64),
                ("capacity", C.c_uint64), ("nslabs", C.c_uint64), ("d_stats", C.c_void_p)]


_lib = None

EXPORTED = (
    "pg_version", "pg_status_string", "pg_table_create", "pg_table_destroy", "pg_table_clear",
    "pg_table_level_info", "pg_table_bytes", "pg_table_set_launch", "pg_table_set_partitioned_insert",
    "pg_bulk_insert", "pg_bulk_insert_with_delete", "pg_bulk_insert_if_not_exists",
    "pg_bulk_insert_if_not_exists_delete", "pg_bulk_query",
    "pg_bulk_remove", "pg_table_count_fill", "pg_table_dump_level", "pg_table_load_level",
    "pg_table_image_bytes", "pg_table_save_image", "pg_table_load_image",
    "pg_host_murmur64a", "pg_host_fastmod", "pg_host_probe_buckets",
    "pg_host_shard_of", "pg_route_by_shard", "pg_scatter_by_perm",
    "pg_slab_create", "pg_slab_destroy", "pg_slab_reset", "pg_slab_info", "pg_slab_bulk_malloc",
    "pg_slab_bulk_free", "pg_slab_count_free", "pg_slab_report", "pg_slab_desc", "pg_slab_set_create", "pg_slab_set_destroy",
    "pg_slab_set_class", "pg_slab_set_bulk_malloc", "pg_slab_set_bulk_free",
    "pg_batch_create", "pg_batch_destroy", "pg_batch_set_launch", "pg_batch_run", "pg_batch_run_static",
    "pg_batch_clear", "pg_table_reserve_insert_scratch", "pg_table_set_fingerprint_residency",
    "pg_pslab_create", "pg_pslab_destroy", "pg_pslab_desc", "pg_pslab_report", "pg_pslab_bulk_malloc",
    "pg_pslab_serial_malloc", "pg_pslab_bulk_free",
    "pg_server_create", "pg_server_destroy", "pg_server_add_table", "pg_server_drop_table", "pg_server_table",
    "pg_server_bytes_in_use", "pg_server_submit", "pg_server_poll", "pg_server_stats", "pg_server_timing",
    "pg_server_add_slab_set", "pg_server_submit_slab",
    "pg_diag_random_access",
)
PG_OP_INSERT, PG_OP_QUERY, PG_OP_REMOVE, PG_OP_INSERT_WITH_DELETE = 0, 1, 2, 3
PG_OP_MALLOC, PG_OP_FREE = 4, 5


def lib() -> C.CDLL:
    """Load libpoggers_b200.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python poggers_b200/build.py`")
    L = C.CDLL(str(LIB_PATH))
    V, P, U64, U32 = C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint32
    L.pg_version.restype = C.c_char_p
    L.pg_status_string.restype = C.c_char_p
    L.pg_status_string.argtypes = [C.c_int]
    L.pg_table_create.restype = C.c_int
    L.pg_table_create.argtypes = [C.POINTER(_TableConfig), U64, C.POINTER(V)]
    L.pg_table_destroy.restype = C.c_int
    L.pg_table_destroy.argtypes = [V]
    L.pg_table_clear.restype = C.c_int
    L.pg_table_clear.argtypes = [V, P]
    L.pg_table_level_info.restype = C.c_int
    L.pg_table_level_info.argtypes = [V, U32, C.POINTER(_LevelInfo)]
    L.pg_table_bytes.restype = U64
    L.pg_table_bytes.argtypes = [V]
    L.pg_table_set_launch.restype = C.c_int
    L.pg_table_set_launch.argtypes = [V, U32, U32, U32, U32]
    L.pg_table_set_partitioned_insert.restype = C.c_int
    L.pg_table_set_partitioned_insert.argtypes = [V, C.c_int]
    L.pg_bulk_insert.restype = C.c_int
    L.pg_bulk_insert.argtypes = [V, P, P, U64, P, P, P]
    L.pg_bulk_query.restype = C.c_int
    L.pg_bulk_query.argtypes = [V, P, U64, P, P, P, P]
    L.pg_bulk_insert_with_delete.restype = C.c_int
    L.pg_bulk_insert_with_delete.argtypes = [V, P, P, U64, P, P, P]
    for f in ("pg_bulk_insert_if_not_exists", "pg_bulk_insert_if_not_exists_delete"):
        getattr(L, f).restype = C.c_int
        getattr(L, f).argtypes = [V, P, P, U64, P, P, P, P, P]
    L.pg_bulk_remove.restype = C.c_int
    L.pg_bulk_remove.argtypes = [V, P, U64, P, P, P]
    L.pg_host_shard_of.restype = U32
    L.pg_host_shard_of.argtypes = [U64, U64, U32]
    L.pg_route_by_shard.restype = C.c_int
    L.pg_route_by_shard.argtypes = [P, P, U32, U64, U32, U64, P, P, P, P, P]
    L.pg_scatter_by_perm.restype = C.c_int
    L.pg_scatter_by_perm.argtypes = [P, P, U64, U32, P, P]
    L.pg_table_image_bytes.restype = U64
    L.pg_table_image_bytes.argtypes = [V]
    L.pg_table_save_image.restype = C.c_int
    L.pg_table_save_image.argtypes = [V, C.c_void_p, U64]
    L.pg_table_load_image.restype = C.c_int
    L.pg_table_load_image.argtypes = [C.c_void_p, U64, C.POINTER(V)]
    L.pg_table_count_fill.restype = C.c_int
    L.pg_table_count_fill.argtypes = [V, U32, P, P]
    L.pg_table_dump_level.restype = C.c_int
    L.pg_table_dump_level.argtypes = [V, U32, P, U64]
    L.pg_table_load_level.restype = C.c_int
    L.pg_table_load_level.argtypes = [V, U32, P, U64]
    L.pg_slab_create.restype = C.c_int
    L.pg_slab_create.argtypes = [U64, U64, C.POINTER(V)]
    L.pg_slab_destroy.restype = C.c_int
    L.pg_slab_destroy.argtypes = [V]
    L.pg_slab_reset.restype = C.c_int
    L.pg_slab_reset.argtypes = [V, P]
    L.pg_slab_info.restype = C.c_int
    L.pg_slab_info.argtypes = [V, C.POINTER(_SlabInfo)]
    L.pg_slab_bulk_malloc.restype = C.c_int
    L.pg_slab_bulk_malloc.argtypes = [V, U64, P, P, P]
    L.pg_slab_bulk_free.restype = C.c_int
    L.pg_slab_bulk_free.argtypes = [V, P, U64, P, P]
    L.pg_slab_count_free.restype = C.c_int
    L.pg_slab_count_free.argtypes = [V, P, P]
    L.pg_slab_report.restype = C.c_int
    L.pg_slab_report.argtypes = [V, C.POINTER(U64), C.POINTER(U64), C.POINTER(U64), C.POINTER(U64)]
    L.pg_slab_set_create.restype = C.c_int
    L.pg_slab_set_create.argtypes = [U32, C.POINTER(U64), C.POINTER(U64), C.POINTER(V)]
    L.pg_slab_set_destroy.restype = C.c_int
    L.pg_slab_set_destroy.argtypes = [V]
    L.pg_slab_set_class.restype = V
    L.pg_slab_set_class.argtypes = [V, U32]
    L.pg_slab_set_bulk_malloc.restype = C.c_int
    L.pg_slab_set_bulk_malloc.argtypes = [V, P, U64, P, P, P]
    L.pg_slab_set_bulk_free.restype = C.c_int
    L.pg_slab_set_bulk_free.argtypes = [V, P, U64, P, P]
    L.pg_batch_create.restype = C.c_int
    L.pg_batch_create.argtypes = [C.POINTER(V), U32, U32, C.POINTER(V)]
    L.pg_batch_destroy.restype = C.c_int
    L.pg_batch_destroy.argtypes = [V]
    L.pg_batch_set_launch.restype = C.c_int
    L.pg_batch_set_launch.argtypes = [V, U32, U32, U32]
    L.pg_batch_run.restype = C.c_int
    L.pg_batch_run.argtypes = [V, P, P, P, P, P, P, P, P]
    L.pg_pslab_create.restype = C.c_int
    L.pg_pslab_create.argtypes = [U64, U64, U32, C.POINTER(V)]
    L.pg_pslab_destroy.restype = C.c_int
    L.pg_pslab_destroy.argtypes = [V]
    L.pg_pslab_desc.restype = C.c_int
    L.pg_pslab_desc.argtypes = [V, P, U64]
    L.pg_pslab_report.restype = C.c_int
    L.pg_pslab_report.argtypes = [V, C.POINTER(U64), C.POINTER(U64), C.POINTER(U64), C.POINTER(U64)]
    L.pg_pslab_bulk_malloc.restype = C.c_int
    L.pg_pslab_bulk_malloc.argtypes = [V, U64, P, P, P]
    L.pg_pslab_serial_malloc.restype = C.c_int
    L.pg_pslab_serial_malloc.argtypes = [V, U32, U32, P, P, P]
    L.pg_pslab_bulk_free.restype = C.c_int
    L.pg_pslab_bulk_free.argtypes = [V, P, U64, P, C.c_int, P]
    L.pg_table_reserve_insert_scratch.restype = C.c_int
    L.pg_table_reserve_insert_scratch.argtypes = [V, U64, P]
    L.pg_table_set_fingerprint_residency.restype = C.c_int
    L.pg_table_set_fingerprint_residency.argtypes = [V, C.c_int]
    L.pg_batch_clear.restype = C.c_int
    L.pg_batch_clear.argtypes = [V, P]
    L.pg_batch_run_static.restype = C.c_int
    L.pg_batch_run_static.argtypes = [C.POINTER(V), U32, P, P, U32, P, P, P, P, P, P]
    L.pg_server_create.restype = C.c_int
    L.pg_server_create.argtypes = [C.POINTER(_ServerConfig), C.POINTER(V)]
    L.pg_server_destroy.restype = C.c_int
    L.pg_server_destroy.argtypes = [V]
    L.pg_server_add_table.restype = C.c_int
    L.pg_server_add_table.argtypes = [V, C.POINTER(_TableConfig), U64, C.POINTER(U32)]
    L.pg_server_drop_table.restype = C.c_int
    L.pg_server_drop_table.argtypes = [V, U32]
    L.pg_server_table.restype = V
    L.pg_server_table.argtypes = [V, U32]
    L.pg_server_add_slab_set.restype = C.c_int
    L.pg_server_add_slab_set.argtypes = [V, U32, P, P, C.POINTER(U32)]
    L.pg_server_submit_slab.restype = C.c_int
    L.pg_server_submit_slab.argtypes = [V, U32, U32, P, U64, P, C.POINTER(U64)]
    L.pg_server_bytes_in_use.restype = U64
    L.pg_server_bytes_in_use.argtypes = [V]
    L.pg_server_submit.restype = C.c_int
    L.pg_server_submit.argtypes = [V, U32, U32, P, P, U64, P, P, C.POINTER(U64)]
    L.pg_server_poll.restype = C.c_int
    L.pg_server_poll.argtypes = [V, U64, C.c_int, C.POINTER(U64), C.POINTER(C.c_double)]
    L.pg_server_stats.restype = C.c_int
    L.pg_server_stats.argtypes = [V, C.POINTER(U64), C.POINTER(U64)]
    L.pg_server_timing.restype = C.c_int
    L.pg_server_timing.argtypes = [V, C.POINTER(_ServerTiming)]
    L.pg_host_murmur64a.restype = U64
    L.pg_host_murmur64a.argtypes = [U64, U64]
    L.pg_host_fastmod.restype = U64
    L.pg_host_fastmod.argtypes = [U64, U64]
    L.pg_host_probe_buckets.restype = U32
    L.pg_host_probe_buckets.argtypes = [C.POINTER(_TableConfig), U32, U64, U64, C.POINTER(U64), U32]
    L.pg_diag_random_access.restype = C.c_int
    L.pg_diag_random_access.argtypes = [P, U64, U32, U64, U64, U32, C.POINTER(U64), P, P]
    _lib = L
    return L


def version() -> str:
    return lib().pg_version().decode()


def status_string(s: int) -> str:
    return lib().pg_status_string(s).decode()


def _check(st: int, what: str) -> None:
    if st != PG_OK:
        raise PoggersError(st, what)


def _ptr(x) -> int | None:
    """Device address of a torch tensor / int / None."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    return x.data_ptr()


def _stream(s) -> int | None:
    if s is None:
        return None
    if isinstance(s, int):
        return s
    return s.cuda_stream


# ---------------------------------------------------------------- configs
@dataclass
class Level:
    nslots: int
    bucket_size: int
    max_probes: int
    scheme: int = SCHEME_BUCKET
    probe: int = PROBE_DOUBLE


@dataclass
class TableConfig:
    format: int
    tile: int
    levels: list[Level] = field(default_factory=list)
    split: bool = False  # PG_TABLE_SPLIT_BUCKETS: keys then values inside each bucket
    fingerprints: bool = False  # PG_TABLE_FINGERPRINTS: L2-resident fingerprint byte per slot

    def c(self) -> _TableConfig:
        c = _TableConfig()
        c.format, c.tile, c.nlevels = self.format, self.tile, len(self.levels)
        c.flags = (PG_TABLE_SPLIT_BUCKETS if self.split else 0) | (PG_TABLE_FINGERPRINTS if self.fingerprints else 0)
        for i, L in enumerate(self.levels):
            c.levels[i] = _LevelConfig(L.nslots, L.bucket_size, L.max_probes, L.scheme, L.probe)
        return c

    def with_sizes(self, *nslots: int) -> "TableConfig":
        if len(nslots) != len(self.levels):
            raise ValueError("sizing lists one slot count per level")
        return TableConfig(self.format, self.tile,
                           [Level(n, L.bucket_size, L.max_probes, L.scheme, L.probe)
                            for n, L in zip(nslots, self.levels)], self.split, self.fingerprints)


class sizing:
    """poggers::sizing::size_in_num_slots<N>: one slot count per table level."""

    class size_in_num_slots:
        def __init__(self, *nslots: int):
            self.nslots = tuple(int(n) for n in nslots)

        def total(self) -> int:
            return sum(self.nslots)


# ---------------------------------------------------------------- table
class Table:
    """One device-resident table (static_table with an optional backing level)."""

    def __init__(self, config: TableConfig, seed: int):
        self.config = config
        self.seed = seed
        self._c = config.c()
        h = C.c_void_p()
        _check(lib().pg_table_create(C.byref(self._c), seed, C.byref(h)), "pg_table_create")
        self._h = h

    @classmethod
    def generate_on_device(cls, config: TableConfig, sizing_obj: "sizing.size_in_num_slots", seed: int) -> "Table":
        """static_table::generate_on_device(Sizing*, seed): raises ValueError when the
        sizing lists a different number of levels (base_table.cuh:116-131)."""
        return cls(config.with_sizes(*sizing_obj.nslots), seed)

    def free_on_device(self) -> None:
        if getattr(self, "_h", None):
            _check(lib().pg_table_destroy(self._h), "pg_table_destroy")
            self._h = None

    def __del__(self):
        try:
            self.free_on_device()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    @property
    def format(self) -> int:
        return self.config.format

    def clear(self, stream=None) -> None:
        _check(lib().pg_table_clear(self._h, _stream(stream)), "pg_table_clear")

    def set_launch(self, block_threads: int = 0, blocks_per_sm: int = 0, max_blocks: int = 0,
                   lanes_per_key: int = 0) -> None:
        _check(lib().pg_table_set_launch(self._h, block_threads, blocks_per_sm, max_blocks, lanes_per_key),
               "pg_table_set_launch")

    def reserve_insert_scratch(self, max_batch_keys: int, stream=None) -> None:
        """Grow the region sort's scratch ahead of time (pg_table_reserve_insert_scratch)."""
        _check(lib().pg_table_reserve_insert_scratch(self._h, max_batch_keys, _stream(stream)),
               "pg_table_reserve_insert_scratch")

    def set_fingerprint_residency(self, resident: bool) -> None:
        """Treat the fingerprint array as L2-resident or not (pg_table_set_fingerprint_residency)."""
        _check(lib().pg_table_set_fingerprint_residency(self._h, int(bool(resident))),
               "pg_table_set_fingerprint_residency")

    def set_partitioned_insert(self, enable: bool) -> None:
        """Region-ordered inserts for large batches (on by default)."""
        _check(lib().pg_table_set_partitioned_insert(self._h, int(bool(enable))), "pg_table_set_partitioned_insert")

    def serial(self, lanes_per_key: int = 0) -> None:
        """One group walks the batch in order (deterministic layout, for parity checks)."""
        lanes = 1 if self.config.fingerprints else (lanes_per_key or self.config.tile)
        if self.format in PACKED_FORMATS:
            lanes = 4 if lanes >= 4 else 1  # the widths the bucketed filter's kernels are built for
        self.set_launch(lanes, 1, 1, lanes)

    def level_info(self, level: int) -> dict:
        info = _LevelInfo()
        _check(lib().pg_table_level_info(self._h, level, C.byref(info)), "pg_table_level_info")
        return {"nbuckets": info.nbuckets, "nslots": info.nslots, "bytes": info.bytes, "seed": info.seed,
                "d_buckets": info.d_buckets}

    def host_bytes_in_use(self) -> int:
        return lib().pg_table_bytes(self._h)

    def bulk_insert(self, keys, vals=None, ok=None, fail_count=None, stream=None, n: int | None = None) -> None:
        n = keys.numel() if n is None else n
        _check(lib().pg_bulk_insert(self._h, _ptr(keys), _ptr(vals), n, _ptr(ok), _ptr(fail_count),
                                    _stream(stream)), "pg_bulk_insert")

    def bulk_query(self, keys, vals_out=None, found=None, hit_count=None, stream=None, n: int | None = None) -> None:
        n = keys.numel() if n is None else n
        _check(lib().pg_bulk_query(self._h, _ptr(keys), n, _ptr(vals_out), _ptr(found), _ptr(hit_count),
                                   _stream(stream)), "pg_bulk_query")

    def bulk_remove(self, keys, ok=None, hit_count=None, stream=None, n: int | None = None) -> None:
        n = keys.numel() if n is None else n
        _check(lib().pg_bulk_remove(self._h, _ptr(keys), n, _ptr(ok), _ptr(hit_count), _stream(stream)),
               "pg_bulk_remove")

    def bulk_insert_with_delete(self, keys, vals=None, ok=None, fail_count=None, stream=None,
                                n: int | None = None) -> None:
        """bucketed_table::insert_with_delete: deleted slots may be reused (packed formats)."""
        n = keys.numel() if n is None else n
        _check(lib().pg_bulk_insert_with_delete(self._h, _ptr(keys), _ptr(vals), n, _ptr(ok), _ptr(fail_count),
                                                _stream(stream)), "pg_bulk_insert_with_delete")

    def bulk_insert_if_not_exists(self, keys, vals=None, vals_out=None, found=None, ok=None, fail_count=None,
                                  stream=None, n: int | None = None, delete: bool = False) -> None:
        """bucketed_table::insert_if_not_exists (delete=True: insert_if_not_exists_delete)."""
        n = keys.numel() if n is None else n
        fn = lib().pg_bulk_insert_if_not_exists_delete if delete else lib().pg_bulk_insert_if_not_exists
        _check(fn(self._h, _ptr(keys), _ptr(vals), n, _ptr(vals_out), _ptr(found), _ptr(ok), _ptr(fail_count),
                  _stream(stream)), "pg_bulk_insert_if_not_exists")

    def count_fill(self, level: int, out, stream=None) -> None:
        """out (2 x uint64 device) += [occupied slots, tombstones] of `level`."""
        _check(lib().pg_table_count_fill(self._h, level, _ptr(out), _stream(stream)), "pg_table_count_fill")

    def get_fill(self, level: int = 0) -> tuple[int, int]:
        import torch
        out = torch.zeros(2, dtype=torch.int64, device="cuda")
        self.count_fill(level, out)
        torch.cuda.synchronize()
        return int(out[0]), int(out[1])

    def dump_level(self, level: int) -> bytes:
        info = self.level_info(level)
        nbytes = info["nslots"] * SLOT_BYTES[self.format]
        buf = C.create_string_buffer(nbytes)
        _check(lib().pg_table_dump_level(self._h, level, buf, nbytes), "pg_table_dump_level")
        return buf.raw

    def save_image(self) -> bytes:
        """Checkpoint image: header + every level in the reference's slot layout."""
        n = lib().pg_table_image_bytes(self._h)
        buf = C.create_string_buffer(n)
        _check(lib().pg_table_save_image(self._h, buf, n), "pg_table_save_image")
        return buf.raw

    def save(self, path) -> None:
        Path(path).write_bytes(self.save_image())

    @classmethod
    def from_image(cls, data: bytes) -> "Table":
        buf = C.create_string_buffer(bytes(data), len(data))
        h = C.c_void_p()
        _check(lib().pg_table_load_image(buf, len(data), C.byref(h)), "pg_table_load_image")
        t = cls.__new__(cls)
        t._h = h
        t.config = _config_from_image(bytes(data))
        t.seed = int.from_bytes(bytes(data[80:88]), "little")
        return t

    @classmethod
    def load(cls, path) -> "Table":
        return cls.from_image(Path(path).read_bytes())

    def load_level(self, level: int, data: bytes) -> None:
        buf = C.create_string_buffer(bytes(data), len(data))
        _check(lib().pg_table_load_level(self._h, level, buf, len(data)), "pg_table_load_level")


def _config_from_image(data: bytes) -> TableConfig:
    """The TableConfig recorded in a checkpoint image's header."""
    c = _TableConfig.from_buffer_copy(data[16:16 + C.sizeof(_TableConfig)])
    levels = [Level(c.levels[i].nslots, c.levels[i].bucket_size, c.levels[i].max_probes, c.levels[i].scheme,
                    c.levels[i].probe) for i in range(c.nlevels)]
    return TableConfig(c.format, c.tile, levels, bool(c.flags & PG_TABLE_SPLIT_BUCKETS),
                       bool(c.flags & PG_TABLE_FINGERPRINTS))


# ---------------------------------------------------------------- named tables
class data_structs:
    """The reference's public aliases (include/poggers/data_structs/) as configurations."""

    @staticmethod
    def tiny_static_table_4(nslots: int) -> TableConfig:
        # static_table<uint64,uint16,dynamic_container<key_val_pair,uint16>,4,4,bucket_insert,20,doubleHasher>
        return TableConfig(FMT_TAGVAL16, 4, [Level(nslots, 4, 20, SCHEME_BUCKET, PROBE_DOUBLE)])

    @staticmethod
    def tcf(nslots: int, backing_nslots: int, tile: int = 4, bucket: int = 16, split: bool = True) -> TableConfig:
        # data_structs/tcf.cuh:30: two-choice shortcut over 16-slot buckets, 2 double-hash probes,
        # backed by tiny_static_table_4.  split: each bucket keeps its tags, then its values
        # (PG_TABLE_SPLIT_BUCKETS), so a probe reads one 32-byte sector of tags; measured on
        # B200 at 0.85 load, inserts + queries 14.6 vs 10.2 G/s at 2^28 slots and 22.1 vs 18.0
        # at 2^22.  Results, dumps and images are the reference's either way.
        return TableConfig(FMT_TAGVAL16, tile, [Level(nslots, bucket, 2, SCHEME_TWO_CHOICE, PROBE_DOUBLE),
                                                Level(backing_nslots, 4, 20, SCHEME_BUCKET, PROBE_DOUBLE)], split)

    @staticmethod
    def tcqf(nslots: int, tile: int = 4, bucket: int = 16) -> TableConfig:
        # tag-only filter: dynamic_container<key_container,uint16> two-choice, no backing
        # (tests/src/bucket_speed_tests.cu:108, tcqf_16_16)
        return TableConfig(FMT_TAG16, tile, [Level(nslots, bucket, 2, SCHEME_TWO_CHOICE, PROBE_DOUBLE)])

    @staticmethod
    def hash_table_64(nslots: int, tile: int = 4, bucket: int = 16, probe: int = PROBE_DOUBLE,
                      max_probes: int = 20) -> TableConfig:
        # data_structs/uint64_hash_table.cuh:35
        return TableConfig(FMT_KV64, tile, [Level(nslots, bucket, max_probes, SCHEME_BUCKET, probe)])

    @staticmethod
    def del_tcf(nslots: int, backing_nslots: int, tile: int = 4, tag_bits: int = 16) -> TableConfig:
        """The bucketed filter with tombstone reuse of tests/src/delete_tests.cu:138-179:
        packed (tag, value) slots, two-choice shortcut over 16-slot buckets with
        XOR power-of-two probing, backed by an 8-slot linear-probing table
        (4000 probes; 400 for 8-bit tags, del_TCF_small)."""
        fmt = FMT_PACKED_TAGVAL16 if tag_bits == 16 else FMT_PACKED_TAGVAL8
        levels = [Level(nslots, 16, 2, SCHEME_TWO_CHOICE_BUCKETED, PROBE_XOR_P2)]
        if backing_nslots:
            levels.append(Level(backing_nslots, 8, 4000 if tag_bits == 16 else 400, SCHEME_LINEAR_BUCKETED,
                                PROBE_LINEAR))
        return TableConfig(fmt, tile, levels)

    @staticmethod
    def two_choice_table_64(nslots: int, tile: int = 4, bucket: int = 8) -> TableConfig:
        # static_table<uint64,uint64,key_val_pair,4,B,power_of_n_insert_shortcut_scheme,2,powerOfTwoHasher>
        return TableConfig(FMT_KV64, tile, [Level(nslots, bucket, 2, SCHEME_TWO_CHOICE, PROBE_P2)])


def diag_random_access(buf, mode: int, accesses: int, seed: int = 1, blocks_per_sm: int = 0, sink=None,
                       stream=None) -> int:
    """pg_diag_random_access over a device buffer (a CUDA tensor, 64-byte
    aligned); returns the exact number of accesses launched."""
    import torch
    if sink is None:
        sink = torch.zeros(1, dtype=torch.int64, device=buf.device)
    done = C.c_uint64(0)
    _check(lib().pg_diag_random_access(_ptr(buf), buf.numel() * buf.element_size(), mode, accesses, seed,
                                       blocks_per_sm, C.byref(done), _ptr(sink), _stream(stream)),
           "pg_diag_random_access")
    return done.value


def host_murmur64a(key: int, seed: int) -> int:
    return lib().pg_host_murmur64a(key, seed)


def host_fastmod(n: int, d: int) -> int:
    return lib().pg_host_fastmod(n, d)


def host_probe_buckets(config: TableConfig, level: int, seed: int, key: int) -> list[int]:
    out = (C.c_uint64 * 64)()
    c = config.c()
    n = lib().pg_host_probe_buckets(C.byref(c), level, seed, key, out, 64)
    return list(out[:n])


# ---------------------------------------------------------------- slab allocator
class allocators:
    """The reference's allocators/ (one_size_slab_allocator) on the slab kernels."""

    class one_size_slab_allocator:
        """Fixed-size objects from slabs of 4096 (allocators/slab_one_size.cuh:58-659)."""

        def __init__(self, num_allocs: int, object_bytes: int):
            h = C.c_void_p()
            _check(lib().pg_slab_create(num_allocs, object_bytes, C.byref(h)), "pg_slab_create")
            self._h = h
            info = _SlabInfo()
            _check(lib().pg_slab_info(h, C.byref(info)), "pg_slab_info")
            self.pool = info.pool
            self.pool_bytes = info.pool_bytes
            self.object_bytes = info.object_bytes
            self.capacity = info.capacity
            self.nslabs = info.nslabs

        @classmethod
        def generate_on_device(cls, num_allocs: int, object_bytes: int):
            return cls(num_allocs, object_bytes)

        def free_on_device(self) -> None:
            if getattr(self, "_h", None):
                _check(lib().pg_slab_destroy(self._h), "pg_slab_destroy")
                self._h = None

        def __del__(self):
            try:
                self.free_on_device()
            except Exception:
                pass

        @property
        def handle(self):
            return self._h

        def reset(self, stream=None) -> None:
            _check(lib().pg_slab_reset(self._h, _stream(stream)), "pg_slab_reset")

        def bulk_malloc(self, ptrs_out, fail_count=None, stream=None, n: int | None = None) -> None:
            """ptrs_out: int64 device tensor receiving one object address (or 0) per slot."""
            n = ptrs_out.numel() if n is None else n
            _check(lib().pg_slab_bulk_malloc(self._h, n, _ptr(ptrs_out), _ptr(fail_count), _stream(stream)),
                   "pg_slab_bulk_malloc")

        def bulk_free(self, ptrs, bad_count=None, stream=None, n: int | None = None) -> None:
            n = ptrs.numel() if n is None else n
            _check(lib().pg_slab_bulk_free(self._h, _ptr(ptrs), n, _ptr(bad_count), _stream(stream)),
                   "pg_slab_bulk_free")

        def report(self) -> dict:
            fs, ms, fo, df = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint64()
            _check(lib().pg_slab_report(self._h, C.byref(fs), C.byref(ms), C.byref(fo), C.byref(df)),
                   "pg_slab_report")
            return {"free_slabs": fs.value, "max_slabs": ms.value, "free_objects": fo.value,
                    "double_frees": df.value}

        def report_fill(self) -> int:
            return self.report()["free_slabs"]

        def report_max(self) -> int:
            return self.report()["max_slabs"]

    class pinned_pool:
        """The reference's slab policy (pg_pslab_*): primary + extra_blocks
        backups pinned per SM, whole-word claims with a per-SM cache, pivot
        and pool.  The template API's one_size_slab_allocator is built on it."""

        def __init__(self, num_allocs: int, object_bytes: int, extra_blocks: int):
            h = C.c_void_p()
            _check(lib().pg_pslab_create(num_allocs, object_bytes, extra_blocks, C.byref(h)), "pg_pslab_create")
            self._h = h

        def free_on_device(self) -> None:
            if getattr(self, "_h", None):
                lib().pg_pslab_destroy(self._h)
                self._h = None

        def __del__(self):
            try:
                self.free_on_device()
            except Exception:
                pass

        def report(self) -> dict:
            v = [C.c_uint64() for _ in range(4)]
            _check(lib().pg_pslab_report(self._h, *[C.byref(x) for x in v]), "pg_pslab_report")
            return {"report_fill": v[0].value, "report_max": v[1].value, "sm_ids": v[2].value,
                    "double_frees": v[3].value}

        def bulk_malloc(self, ptrs_out, fail_count=None, stream=None, n: int | None = None) -> None:
            n = ptrs_out.numel() if n is None else n
            _check(lib().pg_pslab_bulk_malloc(self._h, n, _ptr(ptrs_out), _ptr(fail_count), _stream(stream)),
                   "pg_pslab_bulk_malloc")

        def serial_malloc(self, rounds: int, group: int, ptrs_out, fail_count=None, stream=None) -> None:
            _check(lib().pg_pslab_serial_malloc(self._h, rounds, group, _ptr(ptrs_out), _ptr(fail_count),
                                                _stream(stream)), "pg_pslab_serial_malloc")

        def bulk_free(self, ptrs, counts, serial: bool = False, stream=None, n: int | None = None) -> None:
            """counts (4 x int64, added to): refused, freed, returned to the pool, emptied while pinned."""
            n = ptrs.numel() if n is None else n
            _check(lib().pg_pslab_bulk_free(self._h, _ptr(ptrs), n, _ptr(counts), int(serial), _stream(stream)),
                   "pg_pslab_bulk_free")

    class size_class_set:
        """One pool per size class; each request goes to the smallest class that fits."""

        def __init__(self, class_bytes: list[int], num_allocs: list[int]):
            n = len(class_bytes)
            cb = (C.c_uint64 * n)(*class_bytes)
            na = (C.c_uint64 * n)(*num_allocs)
            h = C.c_void_p()
            _check(lib().pg_slab_set_create(n, cb, na, C.byref(h)), "pg_slab_set_create")
            self._h = h
            self.class_bytes = list(class_bytes)

        def free_on_device(self) -> None:
            if getattr(self, "_h", None):
                _check(lib().pg_slab_set_destroy(self._h), "pg_slab_set_destroy")
                self._h = None

        def __del__(self):
            try:
                self.free_on_device()
            except Exception:
                pass

        def class_report(self, c: int) -> dict:
            a = lib().pg_slab_set_class(self._h, c)
            fs, ms, fo, df = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint64()
            _check(lib().pg_slab_report(a, C.byref(fs), C.byref(ms), C.byref(fo), C.byref(df)), "pg_slab_report")
            info = _SlabInfo()
            _check(lib().pg_slab_info(a, C.byref(info)), "pg_slab_info")
            return {"free_slabs": fs.value, "max_slabs": ms.value, "free_objects": fo.value, "double_frees": df.value,
                    "pool": info.pool, "pool_bytes": info.pool_bytes, "capacity": info.capacity,
                    "object_bytes": info.object_bytes}

        def bulk_malloc(self, sizes, ptrs_out, fail_count=None, stream=None) -> None:
            _check(lib().pg_slab_set_bulk_malloc(self._h, _ptr(sizes), sizes.numel(), _ptr(ptrs_out),
                                                 _ptr(fail_count), _stream(stream)), "pg_slab_set_bulk_malloc")

        def bulk_free(self, ptrs, bad_count=None, stream=None) -> None:
            _check(lib().pg_slab_set_bulk_free(self._h, _ptr(ptrs), ptrs.numel(), _ptr(bad_count), _stream(stream)),
                   "pg_slab_set_bulk_free")


# ---------------------------------------------------------------- multi-table batches
def pack_ops(ops) -> "np.ndarray":
    """[(table, op, offset, count), ...] -> int64 array laid out as pg_op_desc (24 bytes each)."""
    import numpy as np
    a = np.zeros((len(ops), 3), dtype=np.uint64)
    for i, (t, op, off, cnt) in enumerate(ops):
        a[i, 0] = np.uint64(t) | (np.uint64(op) << np.uint64(32))
        a[i, 1] = off
        a[i, 2] = cnt
    return a.view(np.int64).reshape(-1)


class Batch:
    """Tables registered for multi-table runs (pg_batch_*)."""

    def __init__(self, tables: list, max_ops: int):
        arr = (C.c_void_p * len(tables))(*[t.handle.value for t in tables])
        h = C.c_void_p()
        _check(lib().pg_batch_create(arr, len(tables), max_ops, C.byref(h)), "pg_batch_create")
        self._h = h
        self.tables = list(tables)
        self.max_ops = max_ops

    def free(self) -> None:
        if getattr(self, "_h", None):
            _check(lib().pg_batch_destroy(self._h), "pg_batch_destroy")
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def set_launch(self, block_threads: int = 0, blocks_per_sm: int = 0, lanes_per_key: int = 0) -> None:
        _check(lib().pg_batch_set_launch(self._h, block_threads, blocks_per_sm, lanes_per_key), "pg_batch_set_launch")

    def clear(self, stream=None) -> None:
        """Clear every table of the batch with one kernel (pg_batch_clear)."""
        _check(lib().pg_batch_clear(self._h, _stream(stream)), "pg_batch_clear")

    def run(self, ops, nops, keys, vals_in=None, vals_out=None, flags=None, op_counts=None, stream=None) -> None:
        """ops: int64 device tensor from pack_ops; nops: int32 device tensor holding the request count."""
        _check(lib().pg_batch_run(self._h, _ptr(ops), _ptr(nops), _ptr(keys), _ptr(vals_in), _ptr(vals_out),
                                  _ptr(flags), _ptr(op_counts), _stream(stream)), "pg_batch_run")


def batch_run_static(tables: list, ops, nops, max_ops: int, keys, vals_in=None, vals_out=None, flags=None,
                     op_counts=None, stream=None) -> None:
    """pg_batch_run_static: a batch run that allocates no device memory (its
    scratch is a fixed array inside the library; see include/poggers_b200.h)."""
    arr = (C.c_void_p * len(tables))(*[t.handle.value for t in tables])
    _check(lib().pg_batch_run_static(arr, len(tables), _ptr(ops), _ptr(nops), max_ops, _ptr(keys), _ptr(vals_in),
                                     _ptr(vals_out), _ptr(flags), _ptr(op_counts), _stream(stream)),
           "pg_batch_run_static")


# ---------------------------------------------------------------- serving
class Server:
    """Continuous-batching server over resident tables (pg_server_*).

    submit() takes numpy arrays (kept alive until the request is collected);
    poll(rid, wait) returns (count, latency_s) or None while it is running."""

    def __init__(self, hbm_budget_bytes: int, max_wave_keys: int = 1 << 22, max_wave_requests: int = 4096):
        cfg = _ServerConfig(hbm_budget_bytes, max_wave_keys, max_wave_requests, 0)
        h = C.c_void_p()
        _check(lib().pg_server_create(C.byref(cfg), C.byref(h)), "pg_server_create")
        self._h = h
        self._live = {}

    def close(self) -> None:
        if getattr(self, "_h", None):
            _check(lib().pg_server_destroy(self._h), "pg_server_destroy")
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_table(self, config: "TableConfig", seed: int) -> int | None:
        """Table id, or None when the HBM budget is exhausted (PG_ERR_FULL)."""
        c = config.c()
        tid = C.c_uint32()
        st = lib().pg_server_add_table(self._h, C.byref(c), seed, C.byref(tid))
        if st == PG_ERR_FULL:
            return None
        _check(st, "pg_server_add_table")
        return tid.value

    def drop_table(self, tid: int) -> None:
        _check(lib().pg_server_drop_table(self._h, tid), "pg_server_drop_table")

    def bytes_in_use(self) -> int:
        return lib().pg_server_bytes_in_use(self._h)

    def submit(self, tid: int, op: int, keys, vals=None, vals_out=None, flags=None) -> int:
        import numpy as np
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        rid = C.c_uint64()
        _check(lib().pg_server_submit(self._h, tid, op, keys.ctypes.data, None if vals is None else vals.ctypes.data,
                                      len(keys), None if vals_out is None else vals_out.ctypes.data,
                                      None if flags is None else flags.ctypes.data, C.byref(rid)), "pg_server_submit")
        self._live[rid.value] = (keys, vals, vals_out, flags)
        return rid.value

    def add_slab_set(self, class_bytes, num_allocs) -> int | None:
        """A served slab size-class set (pg_slab_set_create); None when the HBM budget is exhausted."""
        cb = (C.c_uint64 * len(class_bytes))(*class_bytes)
        na = (C.c_uint64 * len(num_allocs))(*num_allocs)
        sid = C.c_uint32()
        st = lib().pg_server_add_slab_set(self._h, len(class_bytes), cb, na, C.byref(sid))
        if st == PG_ERR_FULL:
            return None
        _check(st, "pg_server_add_slab_set")
        return sid.value

    def submit_slab(self, sid: int, op: int, data, ptrs_out=None) -> int:
        """PG_OP_MALLOC: data = uint32 sizes, ptrs_out = uint64 array for the
        pointers; PG_OP_FREE: data = uint64 pointers.  Arrays stay alive until polled."""
        import numpy as np
        data = np.ascontiguousarray(data, dtype=np.uint32 if op == PG_OP_MALLOC else np.uint64)
        rid = C.c_uint64()
        _check(lib().pg_server_submit_slab(self._h, sid, op, data.ctypes.data, len(data),
                                           None if ptrs_out is None else ptrs_out.ctypes.data, C.byref(rid)),
               "pg_server_submit_slab")
        self._live[rid.value] = (data, ptrs_out)
        return rid.value

    def poll(self, rid: int, wait: bool = False):
        cnt = C.c_uint64()
        lat = C.c_double()
        st = lib().pg_server_poll(self._h, rid, 1 if wait else 0, C.byref(cnt), C.byref(lat))
        if st == PG_ERR_TIMEOUT:
            return None
        _check(st, "pg_server_poll")
        self._live.pop(rid, None)
        return cnt.value, lat.value

    def stats(self) -> tuple[int, int]:
        w, k = C.c_uint64(), C.c_uint64()
        _check(lib().pg_server_stats(self._h, C.byref(w), C.byref(k)), "pg_server_stats")
        return w.value, k.value

    def timing(self) -> dict:
        """The worker thread's time by stage since creation (pg_server_timing)."""
        t = _ServerTiming()
        _check(lib().pg_server_timing(self._h, C.byref(t)), "pg_server_timing")
        return {f: getattr(t, f) for f, _ in _ServerTiming._fields_}
