"""GPU test of pg_batch_run_static, the batch run that allocates no device memory.

Some callers cannot call cudaMalloc: code that runs inside another memory
allocator, a plugin whose host process owns all device allocations, or a
service whose device memory is fully budgeted ahead of time.  For them the
library keeps the batch run's scratch (the tables' device descriptors, the
per-request chunk offsets and the work counter) in one fixed array compiled
into the library.  This test drives that entry point through the C ABI and
checks that two calls in a row -- inserts, then queries -- give what the
ordinary pg_batch_run gives on an identical set of tables (uint64 tables
exactly, with and without the fingerprint index; the TCF with its backing
level and the bucketed filter without false negatives), that the GPU's free
memory is the same before and after the two calls, and that requests larger
than the fixed array are refused with PG_ERR_TOO_LARGE.

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

from tests.gpu_util import to_dev, u64, val_dtype, vals_np
from poggers_b200 import workload as wl

pytestmark = pytest.mark.gpu

# table kinds the entry point serves with different kernels: uint64 tables
# (plain and with the fingerprint index), the TCF with its backing level, and
# the bucketed filter (packed slots, linear backing level)
KINDS = ["ht", "ht_fingerprints", "tcf_backing", "bucketed_tcf"]


def _config(pg, kind, n):
    if kind.startswith("ht"):
        cfg = pg.data_structs.hash_table_64(n, bucket=8)
        cfg.fingerprints = kind == "ht_fingerprints"
        return cfg
    if kind == "tcf_backing":
        return pg.data_structs.tcf(n, max(n // 100, 64))
    return pg.data_structs.del_tcf(n, n // 100 + 64)


def _tables(pg, sizes, kind="ht"):
    return [pg.Table(_config(pg, kind, n), 300 + i) for i, n in enumerate(sizes)]


class _Call:
    """One batch (one request per table) with every device buffer made up front,
    so that nothing is allocated while the entry point runs."""

    def __init__(self, pg, fmt, reqs, op, vals=None):
        import torch
        keys = np.concatenate(reqs)
        offs = np.concatenate([[0], np.cumsum([len(r) for r in reqs])])
        self.ops = torch.from_numpy(pg.pack_ops([(i, op, int(offs[i]), len(r)) for i, r in enumerate(reqs)])).cuda()
        self.nops = torch.tensor([len(reqs)], dtype=torch.int32, device="cuda")
        self.keys = to_dev(keys)
        self.flags = torch.zeros(len(keys), dtype=torch.uint8, device="cuda")
        self.vout = torch.zeros(len(keys), dtype=val_dtype(fmt), device="cuda") if op == pg.PG_OP_QUERY else None
        self.counts = torch.zeros(len(reqs), dtype=torch.int64, device="cuda")
        self.vin = None if vals is None else to_dev(vals_np(fmt, np.concatenate(vals)))

    def run(self, fn):
        fn(self.ops, self.nops, self.keys, self.vin, self.vout, self.flags, self.counts)

    def results(self):
        vout = np.zeros(len(self.flags), dtype=np.uint64) if self.vout is None else u64(self.vout)
        return self.flags.cpu().numpy(), vout, self.counts.cpu().numpy()


@pytest.mark.parametrize("kind", KINDS)
def test_static_run_equals_allocating_run_on_two_calls(pg, kind):
    import torch
    rng = np.random.default_rng(21)
    sizes = [int(2 ** rng.uniform(12, 16)) for _ in range(40)]
    ins = [wl.keys_without_sentinels(8_000 + i, int(0.6 * n)) for i, n in enumerate(sizes)]
    vals = [wl.values_for(k, 8, 13) for k in ins]
    qry = [np.concatenate([k[: len(k) // 2], wl.keys_without_sentinels(9_000 + i, len(k) - len(k) // 2)])
           for i, k in enumerate(ins)]
    ref_tables = _tables(pg, sizes, kind)
    new_tables = _tables(pg, sizes, kind)
    fmt = ref_tables[0].format
    exact = kind.startswith("ht")  # uint64 tables answer exactly; filters answer by tag
    batch = pg.Batch(ref_tables, max_ops=64)

    def ref_run(ops, nops, keys, vin, vout, flags, counts):
        batch.run(ops, nops, keys, vin, vout, flags, counts)

    def new_run(ops, nops, keys, vin, vout, flags, counts):
        pg.batch_run_static(new_tables, ops, nops, 64, keys, vin, vout, flags, counts)

    offs = np.concatenate([[0], np.cumsum([len(k) for k in ins])])

    def per_request(x, i):
        return x[offs[i]:offs[i + 1]]

    calls = {(w, op): _Call(pg, fmt, ins if op == pg.PG_OP_INSERT else qry, op,
                            vals if op == pg.PG_OP_INSERT else None)
             for w in ("ref", "new") for op in (pg.PG_OP_INSERT, pg.PG_OP_QUERY)}
    empty = torch.zeros(1, dtype=torch.int32, device="cuda")
    calls[("ref", pg.PG_OP_INSERT)].run(ref_run)
    calls[("ref", pg.PG_OP_QUERY)].run(ref_run)
    # an empty batch first: the GPU loads the library's kernels and its fixed
    # array when they are first used, which is device memory the driver takes
    # once, not an allocation by the call
    c0 = calls[("new", pg.PG_OP_INSERT)]
    pg.batch_run_static(new_tables, c0.ops, empty, 64, c0.keys)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    # call 1: inserts; call 2: queries against what call 1 stored (half
    # inserted keys, half absent)
    calls[("new", pg.PG_OP_INSERT)].run(new_run)
    calls[("new", pg.PG_OP_QUERY)].run(new_run)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before, "the calls changed the GPU's free memory"

    a, b = calls[("ref", pg.PG_OP_INSERT)].results(), calls[("new", pg.PG_OP_INSERT)].results()
    placed = (a[0] == 1) & (b[0] == 1)
    assert abs(int((a[0] == 0).sum()) - int((b[0] == 0).sum())) <= 8
    assert placed.mean() > 0.999
    for i in range(len(ins)):
        assert a[2][i] == (per_request(a[0], i) == 0).sum() and b[2][i] == (per_request(b[0], i) == 0).sum()
    qa, qb = calls[("ref", pg.PG_OP_QUERY)].results(), calls[("new", pg.PG_OP_QUERY)].results()
    same = np.zeros(len(qa[0]), dtype=bool)
    positive = np.zeros(len(qa[0]), dtype=bool)
    for i, k in enumerate(ins):
        h = len(k) // 2
        positive[offs[i]:offs[i] + h] = True
        same[offs[i]:offs[i] + h] = per_request(placed, i)[:h]
    if exact:
        same |= ~positive
        assert (qa[0][same] == qb[0][same]).all() and (qa[1][same] == qb[1][same]).all()
        assert (qa[0][same] == positive[same]).all()
    else:
        # no false negatives in either run; absent keys hit only at the filter's
        # false-positive rate (tags of 16 bits: well under 1 %)
        assert qa[0][same].all() and qb[0][same].all()
        assert qa[0][~positive].mean() < 0.01 and qb[0][~positive].mean() < 0.01
    for i in range(len(ins)):
        assert qa[2][i] == per_request(qa[0], i).sum() and qb[2][i] == per_request(qb[0], i).sum()
    batch.free()


def test_static_run_refuses_more_than_its_fixed_scratch(pg):
    import torch
    tables = _tables(pg, [1 << 10] * (pg.PG_STATIC_MAX_TABLES + 1))
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
