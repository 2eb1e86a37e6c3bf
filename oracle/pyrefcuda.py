"""ctypes loader for the reference's CUDA build (oracle/_ref/libpoggers_refcuda.so).

TEST / BASELINE INFRASTRUCTURE: used by tests/golden/make_golden.py to record
golden vectors from the reference itself, by the GPU parity tests, and by
bench.py's reference arm when asked for the reference's CUDA build.  Buffers
are torch CUDA tensors.
"""
from __future__ import annotations

import ctypes as C

from . import pyoracle

KIND_HT_DOUBLE_B8, KIND_HT_ALIAS, KIND_HT_LINEAR_B8, KIND_HT_P2_B8, KIND_TCF, KIND_TCQF, KIND_DEL_TCF, \
    KIND_DEL_TCF_SMALL = range(8)
OP_INSERT, OP_QUERY, OP_REMOVE = 0, 1, 2
# bucketed filters (kinds 6, 7) take these too
OP_INSERT_DELETE, OP_INSERT_IF_NOT_EXISTS, OP_INSERT_IF_NOT_EXISTS_DELETE = 3, 4, 5

_lib = None


def available() -> bool:
    return pyoracle.REFCUDA_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"{pyoracle.REFCUDA_PATH} is missing (make -C oracle refcuda with the reference checkout)")
        L = C.CDLL(str(pyoracle.REFCUDA_PATH))
        V = C.c_void_p
        L.refc_create.restype = V
        L.refc_create.argtypes = [C.c_int, C.c_uint64, C.c_uint64, C.c_uint64]
        L.refc_destroy.argtypes = [V]
        L.refc_bulk.restype = C.c_int
        L.refc_bulk.argtypes = [V, C.c_int, V, V, C.c_uint64, V, V, C.c_int, V]
        L.refc_bbulk.restype = C.c_int
        L.refc_bbulk.argtypes = [V, C.c_int, V, V, C.c_uint64, V, V, V, C.c_int, V]
        L.refc_level.restype = C.c_int
        L.refc_level.argtypes = [V, C.c_int, C.POINTER(V), C.POINTER(C.c_uint64)]
        L.refc_dump.restype = C.c_int
        L.refc_dump.argtypes = [V, C.c_int, V, C.c_uint64]
        _lib = L
    return _lib


def _p(t):
    return None if t is None else t.data_ptr()


class RefTable:
    def __init__(self, kind: int, n0: int, n1: int, seed: int):
        self.kind = kind
        self.h = lib().refc_create(kind, n0, n1, seed)
        if not self.h:
            raise RuntimeError("refc_create failed")

    def close(self):
        if self.h:
            lib().refc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def bulk(self, op, keys, vals=None, flags=None, vals_out=None, serial=False, stream=None):
        st = None if stream is None else stream.cuda_stream
        r = lib().refc_bulk(self.h, op, _p(keys), _p(vals), keys.numel(), _p(flags), _p(vals_out), int(serial), st)
        if r != 0:
            raise RuntimeError("refc_bulk launch failed")

    def bbulk(self, op, keys, vals=None, ok=None, vals_out=None, found=None, serial=False, stream=None):
        """All six operations of the bucketed filters (kinds 6, 7)."""
        st = None if stream is None else stream.cuda_stream
        r = lib().refc_bbulk(self.h, op, _p(keys), _p(vals), keys.numel(), _p(ok), _p(vals_out), _p(found),
                             int(serial), st)
        if r != 0:
            raise RuntimeError("refc_bbulk launch failed")

    # bytes of one bucket per level for the kinds whose levels time_refcuda clears
    # (data_structs::tcf: 16 slots of 4 bytes, backed by tiny_static_table_4's
    # 4 slots of 4 bytes; the 8-slot uint64 table: 8 slots of 16 bytes)
    _BUCKET_BYTES = {KIND_TCF: (64, 16), KIND_TCQF: (32,), KIND_HT_DOUBLE_B8: (128,)}

    def bucket_bytes(self, level: int) -> int:
        return self._BUCKET_BYTES[self.kind][level]

    def level(self, level: int):
        p = C.c_void_p()
        nb = C.c_uint64()
        if lib().refc_level(self.h, level, C.byref(p), C.byref(nb)) != 0:
            raise RuntimeError("refc_level failed")
        return p.value, nb.value

    def dump(self, level: int, nbytes: int) -> bytes:
        buf = C.create_string_buffer(nbytes)
        if lib().refc_dump(self.h, level, buf, nbytes) != 0:
            raise RuntimeError("refc_dump failed")
        return buf.raw
