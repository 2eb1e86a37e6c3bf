"""GPU tests of the sharding kernels (routing by owner, scatter back to batch
order) and of a sharded table on one GPU.  The multi-rank exchange itself is
tested on the host with gloo (tests/test_sharded.py)."""
import numpy as np
import pytest

from tests.gpu_util import to_dev
from poggers_b200 import workload as wl

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nshards", [1, 2, 3, 8, 1024])
@pytest.mark.parametrize("vbytes", [0, 2, 8])
def test_route_by_shard_matches_host_owner(pg, nshards, vbytes):
    import torch
    from poggers_b200.sharded import CudaShardBackend, ROUTE_SEED
    n = 50000
    keys = wl.keys_without_sentinels(3, n)
    dk = to_dev(keys)
    vals = None
    if vbytes == 8:
        vals = torch.arange(n, dtype=torch.int64, device="cuda")
    elif vbytes == 2:
        vals = torch.arange(n, dtype=torch.int32, device="cuda").to(torch.int16)
    b = CudaShardBackend.__new__(CudaShardBackend)
    sk, sv, perm, counts = b.route(dk, vals, nshards, ROUTE_SEED)
    torch.cuda.synchronize()
    f = pg.lib().pg_host_shard_of
    owner = np.array([f(int(k), ROUTE_SEED, nshards) for k in keys])
    assert counts.cpu().numpy().tolist() == np.bincount(owner, minlength=nshards).tolist()
    p = perm.cpu().numpy().astype(np.int64)
    assert sorted(p.tolist()) == list(range(n))
    skn = sk.cpu().numpy().view(np.uint64)
    assert (skn == keys[p]).all()
    assert (np.diff(owner[p]) >= 0).all(), "runs are in shard order"
    if vals is not None:
        assert (sv.cpu().numpy() == vals.cpu().numpy()[p]).all()
    back = b.unpermute(sk, perm)
    assert (back.cpu().numpy().view(np.uint64) == keys).all()


def test_sharded_table_on_one_gpu(pg):
    import torch
    from poggers_b200.sharded import ShardedTable
    cfg = pg.data_structs.hash_table_64(1 << 16, bucket=8)
    st = ShardedTable(cfg, 43)
    keys = wl.keys_without_sentinels(10, 40000)
    vals = wl.values_for(keys, 8, 11)
    ok = st.insert(to_dev(keys), to_dev(vals))
    assert ok.all()
    q = np.concatenate([keys, wl.keys_without_sentinels(12, 5000)])
    f, v = st.query(to_dev(q))
    f = f.cpu().numpy().astype(bool)
    v = v.cpu().numpy().view(np.uint64)
    assert f[:40000].all() and not f[40000:].any()
    assert (v[:40000] == vals).all()
    r = st.remove(to_dev(keys[:10000]))
    assert r.all()
    f2, _ = st.query(to_dev(keys))
    assert not f2[:10000].any() and f2[10000:].all()
    del torch
