"""CPU tests of the C ABI: the library loads, exports every declared symbol,
validates configurations, and its host helpers agree with the oracle.
Nothing here launches a kernel (no GPU needed)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from tests.cases import CASES, product_config
from poggers_b200 import workload as wl

HEADERS = sorted((Path(__file__).resolve().parents[1] / "include").glob("*.h"))


def declared_symbols():
    names = set()
    for h in HEADERS:
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b((?:pg|pgz)_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol(pg):
    names = declared_symbols()
    assert "pg_bulk_insert" in names and len(names) >= 15
    lib = pg.lib()
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(pg.EXPORTED) <= names


def test_version_and_status_strings(pg):
    assert "sm_100a" in pg.version()
    assert pg.status_string(pg.PG_ERR_INVALID) == "invalid argument"


def _create(pg, cfg, seed=1):
    h = C.c_void_p()
    c = cfg.c()
    return pg.lib().pg_table_create(C.byref(c), seed, C.byref(h))


@pytest.mark.parametrize("mut,status", [
    (lambda c: setattr(c, "format", 7), 1),
    (lambda c: setattr(c, "tile", 3), 1),
    (lambda c: setattr(c, "tile", 32), 1),
    (lambda c: c.levels.__setitem__(0, type(c.levels[0])(0, 8, 20, 0, 0)), 1),
    (lambda c: c.levels.__setitem__(0, type(c.levels[0])(64, 8, 0, 0, 0)), 1),
    (lambda c: c.levels.__setitem__(0, type(c.levels[0])(64, 8, 3, 0, 2)), 1),   # p2 needs 2 probes
    (lambda c: c.levels.__setitem__(0, type(c.levels[0])(64, 12, 20, 0, 0)), 4),  # level-0 bucket not compiled
    (lambda c: c.levels.__setitem__(0, type(c.levels[0])(64, 8, 9, 1, 0)), 4),   # two-choice > 4 probes
    (lambda c: setattr(c, "nlevels", 3), 1),
    (lambda c: setattr(c, "flags", 6), 1),
])
def test_create_rejects_bad_configs_before_touching_the_gpu(pg, mut, status):
    cfg = pg.data_structs.hash_table_64(64, bucket=8)
    c = cfg.c()
    mut(c)
    h = C.c_void_p()
    assert pg.lib().pg_table_create(C.byref(c), 1, C.byref(h)) == status
    assert not h.value


def test_null_arguments(pg):
    L = pg.lib()
    assert L.pg_table_destroy(None) == pg.PG_ERR_INVALID
    assert L.pg_bulk_insert(None, None, None, 5, None, None, None) == pg.PG_ERR_INVALID
    assert L.pg_table_bytes(None) == 0


def test_host_murmur_matches_oracle(pg, oracle):
    for k in map(int, wl.splitmix64(5, 2000)):
        for s in (42, 43 * 43):
            assert pg.host_murmur64a(k, s) == oracle.murmur64a(k, s)


def test_fastmod_is_exact(pg):
    rng = np.random.default_rng(0)
    ds = [1, 2, 3, 7, 10, 125, 1000, 10486, 1 << 18, (1 << 23) + 1, (1 << 40) - 3, (1 << 63) + 5, (1 << 64) - 1]
    ds += [int(x) for x in rng.integers(1, 1 << 62, 50, dtype=np.uint64)]
    ns = [0, 1, (1 << 64) - 1, (1 << 63)] + [int(x) for x in wl.splitmix64(9, 300)]
    for d in ds:
        for n in ns:
            assert pg.host_fastmod(n, d) == n % d, (n, d)


@pytest.mark.parametrize("name", sorted(CASES))
def test_probe_buckets_match_oracle(pg, oracle, name):
    cfg, seed = product_config(pg, name)
    fmt = cfg.format
    s = seed
    for lvl, L in enumerate(cfg.levels):
        nb = (L.nslots - 1) // L.bucket_size + 1
        for k in map(int, wl.splitmix64(17, 300)):
            mine = pg.host_probe_buckets(cfg, lvl, seed, k)
            ref = [v % nb for v in oracle.probe_values(L.probe, s, fmt, k, L.max_probes)]
            assert mine == ref
        s = (s * s) % (1 << 64)


def test_load_image_rejects_bad_images_before_touching_the_gpu(pg):
    """A short, foreign or corrupt checkpoint image is refused by the header
    and checksum checks, before any device allocation."""
    lib = pg.lib()
    h = C.c_void_p()
    assert lib.pg_table_load_image(None, 0, C.byref(h)) == pg.PG_ERR_INVALID
    short = C.create_string_buffer(64)
    assert lib.pg_table_load_image(short, 64, C.byref(h)) == pg.PG_ERR_INVALID
    # a well-formed header whose payload checksum does not match
    hdr = bytearray(128)
    hdr[0:8] = b"PGB2TBL1"
    hdr[8:12] = (1).to_bytes(4, "little")
    hdr[12:16] = (128).to_bytes(4, "little")
    cfg = pg.data_structs.hash_table_64(64, bucket=8).c()
    hdr[16:80] = bytes(cfg)
    hdr[88:96] = (64 * 16).to_bytes(8, "little")
    hdr[104:112] = (12345).to_bytes(8, "little")
    img = bytes(hdr) + bytes(64 * 16)
    buf = C.create_string_buffer(img, len(img))
    assert lib.pg_table_load_image(buf, len(img), C.byref(h)) == pg.PG_ERR_INVALID
    # wrong magic
    bad = bytearray(img)
    bad[0] = ord("X")
    buf = C.create_string_buffer(bytes(bad), len(bad))
    assert lib.pg_table_load_image(buf, len(bad), C.byref(h)) == pg.PG_ERR_INVALID
    # payload size disagreeing with the header
    buf = C.create_string_buffer(img[:-16], len(img) - 16)
    assert lib.pg_table_load_image(buf, len(img) - 16, C.byref(h)) == pg.PG_ERR_INVALID
    assert not h.value
