"""Table configurations shared by the oracle tests and the GPU parity tests.

Each golden case (tests/golden/ref_<name>.npz, recorded from the reference's
CUDA build by tests/golden/make_golden.py) names one of the reference's
template tables; CASES maps it to the same table in the oracle's terms and in
the product's terms.
"""
from __future__ import annotations

from pathlib import Path

GOLDEN = Path(__file__).resolve().parent / "golden"

# fmt, partition/tile, [(nslots, bucket, max_probes, scheme, probe), ...], seed
# formats: 0 KV64, 1 TAGVAL16, 2 TAG16; schemes: 0 bucket, 1 two-choice;
# probes: 0 double, 1 linear, 2 power-of-two, 3 xor power-of-two
CASES = {
    "ht_double_b8": (0, 4, [(1000, 8, 20, 0, 0)], 43),
    "ht_alias_b16": (0, 4, [(2048, 16, 20, 0, 0)], 42),
    "ht_linear_b8": (0, 4, [(1000, 8, 20, 0, 1)], 44),
    "ht_p2_b8": (0, 4, [(1000, 8, 2, 1, 2)], 45),
    "tcf": (1, 4, [(2048, 16, 2, 1, 0), (2048 // 100, 4, 20, 0, 0)], 42),
    "tcqf": (2, 4, [(2048, 16, 2, 1, 0)], 42),
}

VAL_BYTES = {0: 8, 1: 2, 2: 0}

# Bucketed filters with tombstone reuse (tests/src/delete_tests.cu:138-179):
# tag bits, [(nslots, bucket, max_probes, scheme, probe), ...], seed.
# schemes: 2 two-choice shortcut over packed buckets, 3 linear over packed buckets
BCASES = {
    "del_tcf": (16, [(4096, 16, 2, 2, 3), (4096 // 100 + 64, 8, 4000, 3, 1)], 42),
    "del_tcf_small": (8, [(4096, 16, 2, 2, 3), (4096 // 100 + 64, 8, 400, 3, 1)], 42),
}


def golden(name: str):
    import numpy as np
    p = GOLDEN / f"ref_{name}.npz"
    if not p.exists():
        return None
    return dict(np.load(p))


def oracle_table(oracle, name: str, partition: int | None = None):
    fmt, tile, levels, seed = CASES[name]
    return oracle.OracleTable(fmt, partition or tile, levels, seed)


def product_config(pg, name: str, tile: int | None = None):
    fmt, t, levels, seed = CASES[name]
    cfg = pg.TableConfig(fmt, tile or t, [pg.Level(*lv) for lv in levels])
    return cfg, seed


def oracle_btable(oracle, name: str):
    bits, levels, seed = BCASES[name]
    return oracle.OracleBucketed(bits, levels, seed)
