"""Device CSR construction (pxr_build_csr) and the device R-MAT sampler
(pxr_rmat_edges) against the host builders in parex_b200/graphs.py: the
same CSR, slot for slot."""
import numpy as np
import pytest
import torch

import parex_b200 as P
from parex_b200 import graphs as G
from parex_b200 import gpu_build as B

pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)).cuda()


def _same(g_dev, g_host):
    np.testing.assert_array_equal(g_dev.offsets.astype(np.int64), g_host.offsets.astype(np.int64))
    np.testing.assert_array_equal(g_dev.cols, g_host.cols)


@pytest.mark.parametrize("scale,abc,seed", [(10, (0.57, 0.19, 0.19), 1), (12, (0.57, 0.19, 0.19), 3),
                                            (11, (0.45, 0.15, 0.15), 7)])
def test_rmat_matches_host_generator(scale, abc, seed):
    off, cols, n, m = B.rmat(scale, 16, *abc, seed=seed)
    host = G.rmat(scale, 16, *abc, seed=seed)
    assert n == host.n and m == host.m
    _same(B.to_host(off, cols), host)


def test_multigraph_with_loops_and_duplicates():
    rng = np.random.default_rng(5)
    n = 5000
    u = rng.integers(0, n, 60000)
    v = rng.integers(0, n, 60000)
    u = np.concatenate([u, v[:1000], np.arange(100)])         # reversed duplicates and self-loops
    v = np.concatenate([v, u[:1000], np.arange(100)])
    off, cols, m = B.build_csr(n, _dev(u), _dev(v))
    host = G.csr_from_edges(u, v, n)
    assert m == host.m
    _same(B.to_host(off, cols), host)


def test_grid_and_empty_cases():
    host = G.grid3d(10)
    src = np.repeat(np.arange(host.n), np.diff(host.offsets.astype(np.int64)))
    off, cols, m = B.build_csr(host.n, _dev(src), _dev(host.cols))   # every edge twice, both ways
    _same(B.to_host(off, cols), host)
    off, cols, m = B.build_csr(7, _dev(np.zeros(0)), _dev(np.zeros(0)))
    assert m == 0 and np.all(off.cpu().numpy() == 0)
    off, cols, m = B.build_csr(3, _dev([0, 1, 2]), _dev([0, 1, 2]))  # only self-loops
    assert m == 0


def test_out_of_range_vertex_is_refused():
    with pytest.raises(P.PxrError):
        B.build_csr(10, _dev([1, 2, 11]), _dev([2, 3, 4]))


def test_device_csr_decomposes_like_host_csr():
    off, cols, n, m = B.rmat(13, 16, seed=2)
    a = P.CudaDeviceManager()
    a.initialize_device(n, m, off.data_ptr(), False, cols.data_ptr())
    a.expanderDecomposition()
    b = P.CudaDeviceManager()
    b.initialize(G.rmat(13, 16, seed=2))
    b.expanderDecomposition()
    np.testing.assert_array_equal(a.getFinalPartition().clusterIds, b.getFinalPartition().clusterIds)


def test_device_sbm_batch_structure_and_decomposition():
    off, cols, n, m, starts = B.sbm_batch(count=10, seed=3, n_lo=200, n_hi=6000, segment_len=1 << 12)
    off2, cols2, n2, m2, starts2 = B.sbm_batch(count=10, seed=3, n_lo=200, n_hi=6000, segment_len=1 << 12)
    g = B.to_host(off, cols)
    np.testing.assert_array_equal(g.cols, B.to_host(off2, cols2).cols)     # deterministic in the seed
    np.testing.assert_array_equal(starts, starts2)
    inst = np.repeat(np.arange(starts.shape[0] - 1), np.diff(starts.astype(np.int64)))
    src = np.repeat(np.arange(n), np.diff(g.offsets.astype(np.int64)))
    assert np.all(inst[src] == inst[g.cols])                                  # no edge leaves its instance
    params = B.sbm_batch_params(count=10, seed=3, n_lo=200, n_hi=6000)
    for i, (ni, blocks, d_in, d_out) in enumerate(params):
        if ni < 2000:
            continue
        lo, hi = int(starts[i]), int(starts[i + 1])
        mean = (g.offsets[hi] - g.offsets[lo]) / ni
        assert abs(mean - (d_in + d_out)) < 0.1 * (d_in + d_out) + 0.5, (i, mean, d_in + d_out)
    # the device-built batch decomposes the same from device and host arrays
    a = P.CudaDeviceManager()
    a.initialize_batched_device(n, m, off.data_ptr(), False, cols.data_ptr(), starts)
    a.expanderDecomposition()
    b = P.CudaDeviceManager()
    b.initialize_batched(g, starts)
    b.expanderDecomposition()
    np.testing.assert_array_equal(a.getFinalPartition().clusterIds, b.getFinalPartition().clusterIds)


def test_device_batch_at_scale_size_independent_properties():
    """A 64-instance device-built batch (about 10 M vertices, mean degree about
    18, so the default components schedule is the sampled one): graph and
    stream drivers and both union-find schedules give the same partition, and
    the device cut-edge count agrees with a host recount of disabled slots.
    (Final ids can join clusters certified in different rounds: certified
    clusters get labels smallest - index - 1, which the reference reuses after
    a round without certificates, and the final partition groups by label as
    the reference's does: a final id may span instances only through such
    labels, which is what is checked here.)"""
    import torch

    off, cols, n, m, starts = B.sbm_batch(count=64, seed=2)
    off64 = off.to(torch.int64)
    ids = []
    for driver, comp in ((P.DRIVER_GRAPH, P.COMPONENTS_AUTO), (P.DRIVER_STREAM, P.COMPONENTS_AUTO),
                         (P.DRIVER_GRAPH, P.COMPONENTS_PLAIN)):
        dm = P.CudaDeviceManager(driver=driver, components=comp)
        dm.initialize_batched_device(n, m, off64.data_ptr(), True, cols.data_ptr(), starts)
        dm.expanderDecomposition()
        fp = dm.getFinalPartition()
        ids.append(fp.clusterIds)
        if len(ids) == 1:
            cut_device = dm.getNumCutEdges()
            final_cols = dm.downloadGraph()[1]
            labels = dm.downloadLabels()
        dm.close()
    np.testing.assert_array_equal(ids[0], ids[1])
    np.testing.assert_array_equal(ids[0], ids[2])
    # a final id that spans two instances only ever groups certified labels
    inst = np.repeat(np.arange(starts.shape[0] - 1), np.diff(starts.astype(np.int64)))
    lo = np.full(ids[0].max() + 1, np.iinfo(np.int64).max, dtype=np.int64)
    hi = np.full(ids[0].max() + 1, -1, dtype=np.int64)
    np.minimum.at(lo, ids[0], inst)
    np.maximum.at(hi, ids[0], inst)
    spans = lo[ids[0]] != hi[ids[0]]
    assert np.all(labels[spans] < 0)
    valid = int(np.count_nonzero(final_cols != 0xFFFFFFFF))
    assert cut_device == m - valid // 2


def test_a_shard_draws_the_same_edges_as_the_whole_batch():
    off, cols, n, m, starts = B.sbm_batch(count=8, seed=5, n_lo=200, n_hi=3000)
    offs, colss, ns, ms, starts_s = B.sbm_batch(count=8, seed=5, n_lo=200, n_hi=3000, instances=[2, 6])
    g, gs = B.to_host(off, cols), B.to_host(offs, colss)

    def rows(graph, lo, hi):
        o = graph.offsets.astype(np.int64)
        return o[lo:hi + 1] - o[lo], graph.cols[o[lo]:o[hi]].astype(np.int64) - lo

    for k, i in enumerate((2, 6)):
        a_off, a_cols = rows(g, int(starts[i]), int(starts[i + 1]))
        b_off, b_cols = rows(gs, int(starts_s[k]), int(starts_s[k + 1]))
        np.testing.assert_array_equal(a_off, b_off)
        np.testing.assert_array_equal(a_cols, b_cols)
