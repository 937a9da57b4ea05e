"""The device planted-partition batch generator (gpu_build.sbm_batch) draws
each instance's size, block count and degrees exactly as the host generator
graphs.sbm_batch does (same per-instance random stream), so the two batches
have the same instances and vertex ranges; only the edge samples differ."""
import numpy as np

from parex_b200 import gpu_build as B
from parex_b200 import graphs as G


def test_device_batch_parameters_match_the_host_generator():
    g, starts = G.sbm_batch(count=6, seed=4, n_lo=50, n_hi=400)
    params = B.sbm_batch_params(count=6, seed=4, n_lo=50, n_hi=400)
    sizes = np.array([p[0] for p in params], dtype=np.int64)
    np.testing.assert_array_equal(np.diff(starts), sizes)
    assert g.n == int(sizes.sum())
    for n, blocks, d_in, d_out in params:
        assert 2 <= blocks <= 64 and blocks <= max(1, n // 2)
        assert 4.0 <= d_in <= 32.0 and 0.1 <= d_out <= 2.0
