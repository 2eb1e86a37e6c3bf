"""GPU test of pg_batch_run_static, the batch run that allocates no device memory.

Some callers cannot call cudaMalloc: code that runs inside another memory
allocator, a plugin whose host process owns all device allocations, or a
service whose device memory is fully budgeted ahead of time.  For them the
library keeps the batch run's scratch (the tables' device descriptors, the
per-request chunk offsets and the work counter) in one fixed array compiled
into the library.  This test drives that entry point through the C ABI and
checks that two calls in a row -- inserts, then queries -- give exactly what
the ordinary pg_batch_run gives on an identical set of tables, and that
requests larger than the fixed array are refused with PG_ERR_TOO_LARGE.

Tolerance, as in the other batch tests: a few inserts can fail even at low
load in small tables (double hashing can cycle over few buckets when the
second hash shares a factor with the bucket count, exactly as in the
reference), and which keys fail depends on the order of concurrent inserts.
So every key that both runs placed must give identical results, each run's
per-request counts must agree with its own flags, and the failure counts of
the two runs may differ by at most a few keys.

It lives in a file that pytest collects last, and passes both on its own in a
fresh process (where its first call looks up the array's device address) and
after the rest of the suite.
"""
import numpy as np
import pytest

from tests.gpu_util import to_dev, u64
from poggers_b200 import workload as wl

pytestmark = pytest.mark.gpu


def _tables(pg, sizes, fingerprints):
    out = []
    for i, n in enumerate(sizes):
        cfg = pg.data_structs.hash_table_64(n, bucket=8)
        cfg.fingerprints = fingerprints
        out.append(pg.Table(cfg, 300 + i))
    return out


def _call(pg, run, reqs, op, vals=None):
    """Run one batch (one request per table) through `run`; return flags, values, counts."""
    import torch
    keys = np.concatenate(reqs)
    offs = np.concatenate([[0], np.cumsum([len(r) for r in reqs])])
    ops = torch.from_numpy(pg.pack_ops([(i, op, int(offs[i]), len(r)) for i, r in enumerate(reqs)])).cuda()
    nops = torch.tensor([len(reqs)], dtype=torch.int32, device="cuda")
    flags = torch.zeros(len(keys), dtype=torch.uint8, device="cuda")
    vout = torch.zeros(len(keys), dtype=torch.int64, device="cuda")
    counts = torch.zeros(len(reqs), dtype=torch.int64, device="cuda")
    vin = None if vals is None else to_dev(np.concatenate(vals))
    run(ops, nops, to_dev(keys), vin, vout if op == pg.PG_OP_QUERY else None, flags, counts)
    torch.cuda.synchronize()
    return flags.cpu().numpy(), u64(vout), counts.cpu().numpy()


@pytest.mark.parametrize("fingerprints", [False, True])
def test_static_run_equals_allocating_run_on_two_calls(pg, fingerprints):
    rng = np.random.default_rng(21)
    sizes = [int(2 ** rng.uniform(12, 16)) for _ in range(40)]
    ins = [wl.keys_without_sentinels(8_000 + i, int(0.6 * n)) for i, n in enumerate(sizes)]
    vals = [wl.values_for(k, 8, 13) for k in ins]
    qry = [np.concatenate([k[: len(k) // 2], wl.keys_without_sentinels(9_000 + i, len(k) - len(k) // 2)])
           for i, k in enumerate(ins)]
    ref_tables = _tables(pg, sizes, fingerprints)
    new_tables = _tables(pg, sizes, fingerprints)
    batch = pg.Batch(ref_tables, max_ops=64)

    def ref_run(ops, nops, keys, vin, vout, flags, counts):
        batch.run(ops, nops, keys, vin, vout, flags, counts)

    def new_run(ops, nops, keys, vin, vout, flags, counts):
        pg.batch_run_static(new_tables, ops, nops, 64, keys, vin, vout, flags, counts)

    offs = np.concatenate([[0], np.cumsum([len(k) for k in ins])])

    def per_request(x, i):
        return x[offs[i]:offs[i + 1]]

    # call 1: inserts
    a = _call(pg, ref_run, ins, pg.PG_OP_INSERT, vals)
    b = _call(pg, new_run, ins, pg.PG_OP_INSERT, vals)
    placed = (a[0] == 1) & (b[0] == 1)
    assert abs(int((a[0] == 0).sum()) - int((b[0] == 0).sum())) <= 8
    assert placed.mean() > 0.999
    for i in range(len(ins)):
        assert a[2][i] == (per_request(a[0], i) == 0).sum() and b[2][i] == (per_request(b[0], i) == 0).sum()
    # call 2: queries against what call 1 stored (half inserted keys, half absent)
    qa = _call(pg, ref_run, qry, pg.PG_OP_QUERY)
    qb = _call(pg, new_run, qry, pg.PG_OP_QUERY)
    same = np.ones(len(qa[0]), dtype=bool)
    for i, k in enumerate(ins):
        h = len(k) // 2
        same[offs[i]:offs[i] + h] = per_request(placed, i)[:h]
    assert (qa[0][same] == qb[0][same]).all() and (qa[1][same] == qb[1][same]).all()
    assert (qa[0][same] == np.concatenate([np.r_[np.ones(len(k) // 2), np.zeros(len(k) - len(k) // 2)]
                                           for k in ins])[same]).all()
    for i in range(len(ins)):
        assert qa[2][i] == per_request(qa[0], i).sum() and qb[2][i] == per_request(qb[0], i).sum()
    batch.free()


def test_static_run_refuses_more_than_its_fixed_scratch(pg):
    import torch
    tables = _tables(pg, [1 << 10] * (pg.PG_STATIC_MAX_TABLES + 1), False)
    ops = torch.zeros(3, dtype=torch.int64, device="cuda")
    nops = torch.zeros(1, dtype=torch.int32, device="cuda")
    keys = torch.zeros(1, dtype=torch.int64, device="cuda")
    with pytest.raises(pg.PoggersError) as e:
        pg.batch_run_static(tables, ops, nops, 1, keys)
    assert e.value.status == pg.PG_ERR_TOO_LARGE
    with pytest.raises(pg.PoggersError) as e:
        pg.batch_run_static(tables[:2], ops, nops, pg.PG_STATIC_MAX_OPS + 1, keys)
    assert e.value.status == pg.PG_ERR_TOO_LARGE
    pg.batch_run_static(tables[:2], ops, nops, pg.PG_STATIC_MAX_OPS, keys)  # an empty batch at the limit is fine
    torch.cuda.synchronize()
