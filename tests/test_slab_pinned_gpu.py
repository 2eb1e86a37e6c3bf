"""GPU parity of the pinned slab pool (the reference's slab policy, behind
pg_pslab_* and the template API's one_size_slab_allocator) against the
oracle's sequential restatement of the reference's allocator
(oracle/poggers_oracle_slabref.c: slab_one_size.cuh:186-506,
offset_slab.cuh:330-1780).

In the serial launch shape -- one warp making malloc() calls of `group` lanes
in order, then one thread freeing in order -- the reference's results are
determined by the sequence: which calls return NULL, what report_fill says
after each phase, and what the free counters count (slabs returned to the pool,
slabs emptied while pinned).  Which objects are handed out is not (the
reference picks bits and words at random), so offsets are checked for being
distinct and inside the pool, not for equality.  At full grid the reference's
own test flow (slab_one_size_tests.cu:220-300: 15M + n + 4096 objects, 15
backups per SM) must hand out every object without a NULL.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
SIZE = 16


def _run_serial(pg, pool, rounds, group):
    import torch
    ptrs = torch.zeros(rounds * group, dtype=torch.int64, device="cuda")
    fails = torch.zeros(1, dtype=torch.int64, device="cuda")
    pool.serial_malloc(rounds, group, ptrs, fails)
    torch.cuda.synchronize()
    return ptrs, int(fails.item())


def _ref_serial(ref, rounds, group):
    nulls, got = 0, []
    for _ in range(rounds):
        o, n = ref.malloc(0, group)
        nulls += n
        got += [int(x) for x in o if x != (1 << 64) - 1]
    return got, nulls


@pytest.mark.parametrize("group,extra", [(32, 1), (7, 1), (1, 0), (32, 3)])
def test_serial_sequence_matches_the_reference_restatement(pg, oracle, group, extra):
    import torch
    probe = pg.allocators.pinned_pool(4096, SIZE, extra)
    sms = probe.report()["sm_ids"]
    probe.free_on_device()
    nslabs = sms * (extra + 1) + 3                    # three slabs left in the pool after the pins
    n = nslabs * 4096
    pool = pg.allocators.pinned_pool(n, SIZE, extra)
    ref = oracle.RefSlab(n, sms=sms, extra_blocks=extra)
    r = pool.report()
    assert r["report_max"] == ref.report_max() == nslabs
    assert r["report_fill"] == ref.report_fill() == 3
    # past exhaustion: the SM's own pins plus the pool's three slabs, then NULLs
    reachable = (extra + 1 + 3) * 4096
    rounds = (reachable + 4096) // group + 1
    ptrs, fails = _run_serial(pg, pool, rounds, group)
    got, nulls = _ref_serial(ref, rounds, group)
    assert fails == nulls, (fails, nulls)
    p = ptrs.cpu().numpy().view(np.uint64)
    live = p[p != 0]
    assert len(live) == len(got) and len(np.unique(live)) == len(live)
    # the pool's three slabs are spent -- unless there is no backup place to
    # refill (extra_blocks 0), in which case the pool is never used
    info_pool = pool.report()
    assert info_pool["report_fill"] == ref.report_fill() == (3 if extra == 0 else 0)
    # free everything in order: the same counts of frees, returned slabs and
    # slabs emptied while pinned as the reference's free_count_misses
    counts = torch.zeros(4, dtype=torch.int64, device="cuda")
    pool.bulk_free(ptrs, counts, serial=True)
    torch.cuda.synchronize()
    codes = [ref.free(x) for x in got]
    c = counts.cpu().numpy()
    assert c[0] == codes.count(oracle.RSLAB_REFUSED) == 0
    assert c[1] == codes.count(oracle.RSLAB_FREED)
    assert c[2] == codes.count(oracle.RSLAB_RETURNED)
    assert c[3] == codes.count(oracle.RSLAB_EMPTIED_PINNED)
    assert pool.report()["report_fill"] == ref.report_fill()
    # a second free of every object changes nothing
    counts.zero_()
    pool.bulk_free(ptrs, counts, serial=True)
    torch.cuda.synchronize()
    assert counts.cpu().numpy()[0] == len(live) and pool.report()["double_frees"] == len(live)
    assert pool.report()["report_fill"] == ref.report_fill()


def test_reference_test_flow_full_grid(pg, oracle):
    """slab_one_size_tests.cu's flow at full grid: 2^20 threads malloc one 16-byte
    object each from a pool of 15M + 2^20 + 4096 objects with 15 backups per SM;
    every malloc succeeds, no object twice, all inside the pool; the pins take
    (E + 1) slabs per SM out of the pool at creation exactly as the restatement
    says; freeing everything refuses nothing and only grows the pool."""
    import torch
    n = 1 << 20
    total = 15000000 + n + 4096
    pool = pg.allocators.pinned_pool(total, SIZE, 15)
    r0 = pool.report()
    ref = oracle.RefSlab(total, sms=r0["sm_ids"], extra_blocks=15)
    assert r0["report_max"] == ref.report_max() and r0["report_fill"] == ref.report_fill()
    ptrs = torch.zeros(n, dtype=torch.int64, device="cuda")
    fails = torch.zeros(1, dtype=torch.int64, device="cuda")
    pool.bulk_malloc(ptrs, fails)
    torch.cuda.synchronize()
    assert int(fails.item()) == 0
    p = ptrs.cpu().numpy().view(np.uint64)
    assert len(np.unique(p)) == n
    r1 = pool.report()
    assert r1["report_fill"] <= r0["report_fill"]
    counts = torch.zeros(4, dtype=torch.int64, device="cuda")
    pool.bulk_free(ptrs, counts)
    torch.cuda.synchronize()
    c = counts.cpu().numpy()
    assert c[0] == 0 and c.sum() == n
    r2 = pool.report()
    assert r1["report_fill"] <= r2["report_fill"] <= r0["report_fill"]
    # returned slabs are exactly those the frees reported
    assert r2["report_fill"] - r1["report_fill"] == c[2]
