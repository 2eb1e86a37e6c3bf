"""CPU tests of the synthetic workload generators."""
import numpy as np

from poggers_b200 import workload as wl


def test_device_splitmix_matches_numpy_stream():
    a = wl.splitmix64(42, 50000, 123)
    b = wl.device_splitmix64(42, 50000, 123, device="cpu").numpy().view(np.uint64)
    assert (a == b).all()


def test_zipf_ranks_are_bounded_and_skewed():
    r = wl.device_zipf_ranks(1 << 20, 200000, 1.1, 3, device="cpu").numpy()
    assert r.min() >= 0 and r.max() < (1 << 20)
    assert (r == 0).mean() > 0.05 and (r < 1000).mean() > 0.5
