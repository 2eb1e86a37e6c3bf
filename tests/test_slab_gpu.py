"""GPU tests of the slab allocator against the sequential pool model.

The reference's own allocator tests check that every malloc of a batch gets a
distinct object inside the pool, that freeing everything restores the fill,
and (the `_bits` variants) catch duplicate allocations with a bitmap
(tests/src/slab_one_size_tests.cu:72-192, 218-308).  Object identities depend
on which SM ran which warp, in the reference too, so parity here is on those
invariants and on every count, which the sequential model
(oracle/poggers_oracle.c, pgo_slab_*) fixes exactly.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _offsets(a, ptrs):
    p = ptrs.cpu().numpy().view(np.uint64)
    ok = p != 0
    off = (p[ok] - np.uint64(a.pool)) // np.uint64(a.object_bytes)
    rem = (p[ok] - np.uint64(a.pool)) % np.uint64(a.object_bytes)
    return ok, off, rem


@pytest.mark.parametrize("num_allocs,size", [(4096, 16), (10000, 64), (1 << 20, 8), (3 * 4096 + 5, 4096)])
def test_malloc_distinct_in_pool_and_free_restores(pg, oracle, num_allocs, size):
    import torch
    a = pg.allocators.one_size_slab_allocator(num_allocs, size)
    o = oracle.OracleSlab(num_allocs)
    assert a.capacity == o.capacity
    n = num_allocs
    ptrs = torch.zeros(n, dtype=torch.int64, device="cuda")
    fails = torch.zeros(1, dtype=torch.int64, device="cuda")
    a.bulk_malloc(ptrs, fails)
    torch.cuda.synchronize()
    ok, off, rem = _offsets(a, ptrs)
    _, ofails = o.malloc(n)
    assert int(fails.item()) == ofails == int((~ok).sum())
    assert (rem == 0).all() and (off < a.capacity).all()
    assert len(np.unique(off)) == len(off), "an object was handed out twice"
    rep = a.report()
    assert rep["free_objects"] == o.free_objects == a.capacity - len(off)
    # free everything: the pool is whole again
    bad = torch.zeros(1, dtype=torch.int64, device="cuda")
    a.bulk_free(ptrs, bad)
    torch.cuda.synchronize()
    assert int(bad.item()) == 0
    rep = a.report()
    assert rep["free_objects"] == a.capacity and rep["free_slabs"] == rep["max_slabs"] == a.nslabs
    assert rep["double_frees"] == 0


def test_exhaustion_fails_exactly_past_capacity(pg, oracle):
    import torch
    a = pg.allocators.one_size_slab_allocator(8192, 32)
    n = 8192 + 1000
    ptrs = torch.zeros(n, dtype=torch.int64, device="cuda")
    fails = torch.zeros(1, dtype=torch.int64, device="cuda")
    a.bulk_malloc(ptrs, fails)
    torch.cuda.synchronize()
    ok, off, _ = _offsets(a, ptrs)
    assert int(fails.item()) == 1000 and ok.sum() == 8192
    assert len(np.unique(off)) == 8192


def test_churn_free_half_then_remalloc(pg, oracle):
    """Config-5 style churn on one class: malloc all, free a seeded random half,
    malloc again; live objects never collide and counts match the model."""
    import torch
    from poggers_b200 import workload as wl
    cap_req = 1 << 18
    a = pg.allocators.one_size_slab_allocator(cap_req, 48)
    o = oracle.OracleSlab(cap_req)
    n = cap_req - 1000
    ptrs = torch.zeros(n, dtype=torch.int64, device="cuda")
    a.bulk_malloc(ptrs)
    oo, _ = o.malloc(n)
    half = wl.fisher_yates_half(n, 9)
    idx = torch.from_numpy(half).cuda()
    freed = ptrs[idx].contiguous()
    bad = torch.zeros(1, dtype=torch.int64, device="cuda")
    a.bulk_free(freed, bad)
    assert o.free(oo[half]) == 0
    keep = np.ones(n, dtype=bool)
    keep[half] = False
    m = len(half) + 500
    again = torch.zeros(m, dtype=torch.int64, device="cuda")
    fails = torch.zeros(1, dtype=torch.int64, device="cuda")
    a.bulk_malloc(again, fails)
    torch.cuda.synchronize()
    _, ofails = o.malloc(m)
    assert int(bad.item()) == 0
    assert int(fails.item()) == ofails
    live = np.concatenate([ptrs.cpu().numpy()[keep], again.cpu().numpy()])
    live = live[live != 0]
    assert len(np.unique(live)) == len(live), "a live object was handed out again"
    assert a.report()["free_objects"] == o.free_objects


def test_double_free_and_foreign_pointers_are_counted(pg):
    import torch
    a = pg.allocators.one_size_slab_allocator(4096, 64)
    ptrs = torch.zeros(100, dtype=torch.int64, device="cuda")
    a.bulk_malloc(ptrs)
    bad = torch.zeros(1, dtype=torch.int64, device="cuda")
    a.bulk_free(ptrs[:10].contiguous(), bad)
    a.bulk_free(ptrs[:10].contiguous(), bad)             # double free
    junk = torch.tensor([a.pool + 3, a.pool + a.pool_bytes + 64, 0], dtype=torch.int64, device="cuda")
    a.bulk_free(junk, bad)                                # misaligned, outside, NULL (skipped)
    torch.cuda.synchronize()
    assert int(bad.item()) == 12
    rep = a.report()
    assert rep["double_frees"] == 10
    assert rep["free_objects"] == a.capacity - 90


def test_size_classes_route_to_the_smallest_fitting_class(pg):
    import torch
    classes = [16 << i for i in range(9)]  # 16 .. 4096 bytes
    s = pg.allocators.size_class_set(classes, [1 << 14] * 9)
    rng = np.random.default_rng(5)
    sizes = np.exp(rng.uniform(np.log(16), np.log(4096), 50000)).astype(np.uint32)
    sizes = np.concatenate([sizes, np.array([1, 16, 17, 4096, 4097], dtype=np.uint32)])
    d_sizes = torch.from_numpy(sizes.view(np.int32)).cuda()
    ptrs = torch.zeros(len(sizes), dtype=torch.int64, device="cuda")
    fails = torch.zeros(1, dtype=torch.int64, device="cuda")
    s.bulk_malloc(d_sizes, ptrs, fails)
    torch.cuda.synchronize()
    p = ptrs.cpu().numpy().view(np.uint64)
    assert int(fails.item()) == 1 and p[-1] == 0          # 4097 bytes fits no class
    want = np.searchsorted(np.array(classes), sizes)      # smallest class >= size
    for c in range(9):
        r = s.class_report(c)
        sel = (want == c) & (p != 0)
        pc = p[sel]
        assert ((pc >= np.uint64(r["pool"])) & (pc < np.uint64(r["pool"] + r["pool_bytes"]))).all()
        assert ((pc - np.uint64(r["pool"])) % np.uint64(r["object_bytes"]) == 0).all()
        assert len(np.unique(pc)) == len(pc)
        assert r["free_objects"] == r["capacity"] - len(pc)
    bad = torch.zeros(1, dtype=torch.int64, device="cuda")
    s.bulk_free(ptrs, bad)
    torch.cuda.synchronize()
    assert int(bad.item()) == 0
    assert all(s.class_report(c)["free_objects"] == s.class_report(c)["capacity"] for c in range(9))
