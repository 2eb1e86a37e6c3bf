"""Launch-shape autotuner for the bulk kernels.

The reference tunes its tile and bucket sizes by hand with separate test
programs (tests/src/power_2_tests.cu:338-430, tests/src/test_cg_variations.cu:
878-1040 sweep tile sizes 1-32 against bucket sizes 8-64).  Here the sweep is a
library function: for one table shape it times bulk insert and bulk query on
the device over

  * lanes per key (the tile: 1, 2, 4, 8, 16; results do not depend on it,
    because filled slots always form a prefix of each bucket),
  * threads per block and resident blocks per SM,
  * optionally the bucket size (which does change the table, and so is only
    swept when the caller allows it),

and returns the fastest shape.  Results are cached per GPU and table shape in
a JSON file so a serving process pays for the sweep once.

The multi-table batch path (pg_batch_run over many tables of uneven size) has
its own sweep: lanes per key (1, 2, 4, 8, 16), bucket size (8, 16, 32: a
different table, built once per bucket size) and resident blocks per SM, each
shape timed as replays of one captured CUDA graph holding the batch's insert
run and query run, with the batch cleared by one kernel between replays.
The pick is the fastest shape among those whose insert failures are within
a small margin of the fewest any shape had (small two-choice tables fail
more keys when too many of their keys are in flight at once).  Cached per GPU
and size class of the batch.
"""
from __future__ import annotations

import itertools
import json
import os
import time
from dataclasses import asdict, dataclass
from pathlib import Path

import numpy as np

CACHE = Path(os.environ.get("POGGERS_B200_TUNE_CACHE", str(Path.home() / ".cache" / "poggers_b200_tune.json")))


@dataclass
class Shape:
    tile: int
    block_threads: int
    blocks_per_sm: int
    bucket: int
    split: bool = False


@dataclass
class Result:
    shape: Shape
    insert_ms: float
    query_ms: float

    @property
    def total_ms(self) -> float:
        return self.insert_ms + self.query_ms


def _dev(a: np.ndarray):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64 if a.dtype == np.uint64 else np.int16)).cuda()


def time_shape(make_config, shape: Shape, seed: int, keys, vals, qkeys, reps: int = 3) -> Result:
    """Median device time of one bulk insert (into a cleared table) and one bulk query."""
    import torch
    import poggers_b200 as pg

    cfg = make_config(shape.tile, shape.bucket)
    cfg.split = shape.split
    t = pg.Table(cfg, seed)
    t.set_launch(shape.block_threads, shape.blocks_per_sm, 0, shape.tile)
    s = torch.cuda.current_stream()
    ins, qry = [], []
    for _ in range(reps + 1):
        t.clear(s)
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(s)
        t.bulk_insert(keys, vals, None, None, s)
        e1.record(s)
        t.bulk_query(qkeys, None, None, None, s)
        e2.record(s)
        torch.cuda.synchronize()
        ins.append(e0.elapsed_time(e1))
        qry.append(e1.elapsed_time(e2))
    t.free_on_device()
    return Result(shape, float(np.median(ins[1:])), float(np.median(qry[1:])))


def sweep(make_config, seed: int, keys, vals, qkeys, tiles=(1, 2, 4, 8), block_threads=(128, 256),
          blocks_per_sm=(4, 8, 16), buckets=(None,), splits=(False,), reps: int = 3) -> list[Result]:
    """Time every shape of the grid; `make_config(tile, bucket)` builds the table
    configuration (bucket None = the table's own bucket size)."""
    out = []
    for tile, bt, bps, b, d in itertools.product(tiles, block_threads, blocks_per_sm, buckets, splits):
        bucket = b if b is not None else make_config(1, None).levels[0].bucket_size
        if tile > bucket or bt % tile:
            continue
        out.append(time_shape(make_config, Shape(tile, bt, bps, bucket, d), seed, keys, vals, qkeys, reps))
    return out


def best(results: list[Result]) -> Result:
    return min(results, key=lambda r: r.total_ms)


def _read_cache() -> dict:
    """The tuning cache, or an empty one when the file is missing or unreadable
    (a write cut short by another process): the sweep then runs again."""
    try:
        return json.loads(CACHE.read_text()) if CACHE.exists() else {}
    except (OSError, ValueError):
        return {}


def cache_key(gpu_name: str, config) -> str:
    L = config.levels[0]
    fp = int(bool(getattr(config, "fingerprints", False)))
    return (f"{gpu_name}|fmt{config.format}|b{L.bucket_size}|s{L.scheme}|p{L.probe}|n{L.nslots.bit_length()}"
            f"|lv{len(config.levels)}|fp{fp}")


def tuned_shape(config, seed: int, keys, vals, qkeys, **grid) -> Shape:
    """The cached best shape for this GPU and table shape, sweeping on a miss."""
    import torch
    name = torch.cuda.get_device_name()
    key = cache_key(name, config)
    cache = _read_cache()
    if key in cache:
        return Shape(**cache[key]["shape"])

    def make(tile, bucket):
        import poggers_b200 as pg
        lv = [pg.Level(l.nslots, l.bucket_size if (i or bucket is None) else bucket, l.max_probes, l.scheme, l.probe)
              for i, l in enumerate(config.levels)]
        return pg.TableConfig(config.format, tile, lv, getattr(config, "split", False),
                              getattr(config, "fingerprints", False))

    res = sweep(make, seed, keys, vals, qkeys, **grid)
    b = best(res)
    cache[key] = {"shape": asdict(b.shape), "insert_ms": b.insert_ms, "query_ms": b.query_ms, "when": time.time()}
    CACHE.parent.mkdir(parents=True, exist_ok=True)
    CACHE.write_text(json.dumps(cache, indent=1))
    return b.shape


# ---------------------------------------------------------------- batch path
@dataclass
class BatchShape:
    lanes: int
    bucket: int
    blocks_per_sm: int
    block_threads: int = 256


@dataclass
class BatchResult:
    shape: BatchShape
    step_ms: float        # one graph replay: every insert request, then every query request
    insert_failures: int


def _batch_ok(results: list[BatchResult]) -> list[BatchResult]:
    fewest = min(r.insert_failures for r in results)
    bound = fewest + max(16, fewest // 2)
    return [r for r in results if r.insert_failures <= bound]


def best_batch(results: list[BatchResult]) -> BatchResult:
    return min(_batch_ok(results), key=lambda r: r.step_ms)


def sweep_batch(make_configs, seeds, ins_ops, q_ops, nops, keys, vals, qkeys, lanes=(1, 2, 4, 8, 16),
                buckets=(8, 16, 32), blocks_per_sm=(4, 8, 16), reps: int = 3) -> list[BatchResult]:
    """Time every batch shape.  make_configs(bucket) -> one TableConfig per
    table; ins_ops / q_ops are device request arrays (pack_ops) over keys /
    qkeys, nops a device int32 holding the request count."""
    import torch
    import poggers_b200 as pg

    out = []
    n = keys.numel()
    ok = torch.zeros(n, dtype=torch.uint8, device=keys.device)
    found = torch.zeros(qkeys.numel(), dtype=torch.uint8, device=keys.device)
    s = torch.cuda.Stream()
    for bucket in buckets:
        tables = [pg.Table(c, sd) for c, sd in zip(make_configs(bucket), seeds)]
        batch = pg.Batch(tables, max_ops=max(1, len(tables)))
        for ln, bps in itertools.product(lanes, blocks_per_sm):
            if ln > bucket:
                continue
            try:
                batch.set_launch(256, bps, ln)
            except pg.PoggersError:
                continue
            g = torch.cuda.CUDAGraph()
            with torch.cuda.stream(s):
                batch.clear(s)
                batch.run(ins_ops, nops, keys, vals, None, ok, None, s)
                batch.run(q_ops, nops, qkeys, None, None, found, None, s)
            s.synchronize()
            with torch.cuda.graph(g, stream=s):
                batch.run(ins_ops, nops, keys, vals, None, ok, None, s)
                batch.run(q_ops, nops, qkeys, None, None, found, None, s)
            times = []
            for _ in range(reps + 1):
                with torch.cuda.stream(s):
                    batch.clear(s)
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(s)
                    g.replay()
                    e1.record(s)
                s.synchronize()
                times.append(e0.elapsed_time(e1))
            fails = int((ok == 0).sum().item())
            out.append(BatchResult(BatchShape(ln, bucket, bps), float(np.median(times[1:])), fails))
            del g
        batch.free()
        for t in tables:
            t.free_on_device()
    return out


def batch_cache_key(gpu_name: str, configs) -> str:
    c0 = configs[0]
    L = c0.levels[0]
    lo = min(c.levels[0].nslots for c in configs).bit_length()
    hi = max(c.levels[0].nslots for c in configs).bit_length()
    return (f"{gpu_name}|batch|fmt{c0.format}|s{L.scheme}|p{L.probe}|lv{len(c0.levels)}|t{len(configs).bit_length()}"
            f"|n{lo}-{hi}")


def tuned_batch_shape(make_configs, seeds, ins_ops, q_ops, nops, keys, vals, qkeys, **grid):
    """The cached best batch shape for this GPU and size class, sweeping on a
    miss.  Returns (shape, results of the sweep or None when cached)."""
    import torch
    key = batch_cache_key(torch.cuda.get_device_name(), make_configs(16))
    cache = _read_cache()
    if key in cache:
        return BatchShape(**cache[key]["shape"]), None
    res = sweep_batch(make_configs, seeds, ins_ops, q_ops, nops, keys, vals, qkeys, **grid)
    b = best_batch(res)
    cache[key] = {"shape": asdict(b.shape), "step_ms": b.step_ms, "insert_failures": b.insert_failures,
                  "when": time.time()}
    CACHE.parent.mkdir(parents=True, exist_ok=True)
    CACHE.write_text(json.dumps(cache, indent=1))
    return b.shape, res
