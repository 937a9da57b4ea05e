"""Batched independent instances (pxr_initialize_batched): every instance
starts as its own cluster and the whole batch advances through shared rounds.

The oracle is given the same starting state (labels = instance index, every
vertex active in vertex order, the product's seeded potentials) and must agree
bit for bit per stage and end to end; no output cluster may span two
instances; malformed batches are refused.
"""
import numpy as np
import pytest

import parex_b200 as P
from parex_b200 import graphs as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _bits(x):
    return np.asarray(x, dtype=np.float32).view(np.uint32)


def _batch(count=14, seed=5, n_lo=20, n_hi=3000):
    g, starts = G.sbm_batch(count=count, seed=seed, n_lo=n_lo, n_hi=n_hi)
    # append tiny instances: a single vertex, an edge, two disjoint triangles
    n0 = g.n
    extra_edges = [(n0 + 1, n0 + 2), (n0 + 3, n0 + 4), (n0 + 4, n0 + 5), (n0 + 3, n0 + 5),
                   (n0 + 6, n0 + 7), (n0 + 7, n0 + 8), (n0 + 6, n0 + 8)]
    src = np.repeat(np.arange(g.n, dtype=np.int64), np.diff(g.offsets.astype(np.int64)))
    keep = src < g.cols
    u = np.concatenate([src[keep], [a for a, _ in extra_edges]])
    v = np.concatenate([g.cols[keep].astype(np.int64), [b for _, b in extra_edges]])
    n = n0 + 9
    full = G.csr_from_edges(u, v, n, "batch")
    starts = np.concatenate([starts, [n0 + 1, n0 + 3, n]]).astype(np.uint32)
    return full, starts


def _oracle_for(dm, g, starts):
    k = starts.shape[0] - 1
    labels = np.repeat(np.arange(k, dtype=np.int32), np.diff(starts.astype(np.int64)))
    act = np.zeros(g.n, dtype=O.LNODE)
    act["nix"] = np.arange(g.n, dtype=np.uint32)
    act["label"] = labels
    orc = O.Oracle(g.offsets, g.cols, O.MODE_PXR)
    orc.set_state(labels, act, dm.readRandomWalkValues().astype(np.float64),
                  np.diff(g.offsets.astype(np.int64)).astype(np.uint32), g.cols, k, 0)
    return orc, labels


def test_batched_stages_match_oracle():
    g, starts = _batch()
    dm = P.CudaDeviceManager(driver=P.DRIVER_STREAM)
    dm.initialize_batched(g, starts)
    orc, _ = _oracle_for(dm, g, starts)
    assert dm.getNumClusters() == starts.shape[0] - 1
    np.testing.assert_array_equal(dm.downloadLabels(), orc.labels())
    for _ in range(6):
        orc.walk()
        dm.iterateRandomWalk()
        np.testing.assert_array_equal(_bits(dm.readRandomWalkValues()), _bits(orc.potentials()))
        orc.sweep()
        dm.computeSweepCuts()
        part, srt = dm.downloadPartition(), orc.sorted()
        np.testing.assert_array_equal(part["nix"], srt["nix"])
        np.testing.assert_array_equal(part["prefix_volume"], srt["prefix_volume"])
        np.testing.assert_array_equal(part["prefix_edge_diff"], srt["prefix_edge_diff"])
        cuts, oc = dm.readSweepCuts(), orc.all_cuts()
        np.testing.assert_array_equal(cuts.cuts["offset"], oc["offset"])
        np.testing.assert_array_equal(_bits(cuts.cuts["sparsity"]), _bits(oc["sparsity"]))
        orc.cut_clusters()
        dm.cutClusters()
        np.testing.assert_array_equal(dm.downloadLabels(), orc.labels())
        np.testing.assert_array_equal(dm.downloadDegrees(), orc.internal_degrees())
        np.testing.assert_array_equal(dm.downloadGraph()[1], orc.cols())


@pytest.mark.parametrize("driver", [P.DRIVER_GRAPH, P.DRIVER_STREAM])
def test_batched_end_to_end(driver):
    g, starts = _batch(count=24, seed=9, n_lo=10, n_hi=5000)
    dm = P.CudaDeviceManager(driver=driver)
    dm.initialize_batched(g, starts)
    orc, inst = _oracle_for(dm, g, starts)
    dm.expanderDecomposition()
    orc.decompose()
    fp = dm.getFinalPartition()
    ids, k = orc.final_partition()
    np.testing.assert_array_equal(fp.clusterIds, ids)
    assert fp.numClusters == k
    assert dm.getNumCutEdges() == orc.num_cut_edges()
    # no cluster spans two instances
    owner = np.full(k, -1, dtype=np.int64)
    first = np.unique(fp.clusterIds, return_index=True)[1]
    owner[fp.clusterIds[first]] = inst[first]
    np.testing.assert_array_equal(owner[fp.clusterIds], inst)


def test_batched_rejects_malformed():
    g, starts = _batch(count=3, seed=1, n_lo=20, n_hi=50)
    dm = P.CudaDeviceManager()
    with pytest.raises(P.PxrError):
        dm.initialize_batched(g, starts[:-1])                 # does not end at n
    bad = starts.copy()
    bad[2] = bad[1]
    with pytest.raises(P.PxrError):
        dm.initialize_batched(g, bad)                         # empty instance
    # an edge between the first two instances
    src = np.repeat(np.arange(g.n, dtype=np.int64), np.diff(g.offsets.astype(np.int64)))
    keep = src < g.cols
    u = np.concatenate([src[keep], [int(starts[0])]])
    v = np.concatenate([g.cols[keep].astype(np.int64), [int(starts[1])]])
    joined = G.csr_from_edges(u, v, g.n)
    with pytest.raises(P.PxrError):
        dm.initialize_batched(joined, starts)
    dm.initialize_batched(g, starts)                          # still usable
    dm.expanderDecomposition()


def test_batched_components_schedules_agree_with_the_oracle():
    """The sampled union-find schedule on a batch with a one-vertex instance,
    a one-edge instance and an instance of two disjoint triangles: the same
    decomposition as the oracle's (representatives are per split cluster,
    so instances never share one)."""
    g, starts = _batch(count=10, seed=3, n_lo=10, n_hi=2000)
    out = []
    for comp in (P.COMPONENTS_PLAIN, P.COMPONENTS_SAMPLED):
        dm = P.CudaDeviceManager(components=comp)
        dm.initialize_batched(g, starts)
        if not out:
            orc, _ = _oracle_for(dm, g, starts)
        dm.expanderDecomposition()
        out.append((dm.getFinalPartition(), dm.getNumCutEdges()))
    orc.decompose()
    ids, k = orc.final_partition()
    for fp, cut in out:
        np.testing.assert_array_equal(fp.clusterIds, ids)
        assert fp.numClusters == k
        assert cut == orc.num_cut_edges()
