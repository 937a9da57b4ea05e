"""CUDA product vs the CPU oracle in its product-arithmetic mode (ORC_MODE_PXR).

Both run the same algorithm with the same operation sequence, so every output
is compared bit for bit: potentials (float bits), sweep order and prefix sums,
per-cluster argmin, labels, internal degrees, disabled CSR slots, final
partition and cut counts - per stage for every round and end to end.  The
product is driven through the C ABI (parex_b200.CudaDeviceManager).
"""
import numpy as np
import pytest

import parex_b200 as P
from parex_b200 import graphs as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _edges_graph(n, edges):
    e = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
    if e.size == 0:
        return G.CSRGraph(np.zeros(n + 1, dtype=np.uint32), np.zeros(0, dtype=np.uint32), "empty")
    return G.csr_from_edges(e[:, 0], e[:, 1], n)


SMALL = {
    "sbm2k": lambda: G.sbm_graph(2048, 8, 10.0, 0.5, 7),
    "grid16": lambda: G.grid3d(16),
    "rmat11": lambda: G.rmat(11, 16, seed=3),
    "regular8": lambda: G.random_regular(1024, 8, seed=2),
    "two_triangles": lambda: _edges_graph(6, [(0, 1), (1, 2), (0, 2), (3, 4), (4, 5), (3, 5)]),
    "path": lambda: _edges_graph(64, [(i, i + 1) for i in range(63)]),
    "star": lambda: _edges_graph(33, [(0, i) for i in range(1, 33)]),
    "complete8": lambda: _edges_graph(8, [(i, j) for i in range(8) for j in range(i + 1, 8)]),
    "isolated": lambda: _edges_graph(10, [(0, 1), (2, 3)]),
    "no_edges": lambda: _edges_graph(5, []),
    "single": lambda: _edges_graph(1, []),
}


def _bits(x):
    return np.asarray(x, dtype=np.float32).view(np.uint32)


def _pair(g, **kw):
    dm = P.CudaDeviceManager(driver=P.DRIVER_STREAM, **kw)
    dm.initialize(g)
    orc = O.Oracle(g.offsets, g.cols, O.MODE_PXR)
    orc.set_potentials(dm.readRandomWalkValues().astype(np.float64))
    return dm, orc


def _check_round(dm, orc):
    orc.walk()
    dm.iterateRandomWalk()
    np.testing.assert_array_equal(_bits(dm.readRandomWalkValues()), _bits(orc.potentials()))
    orc.sweep()
    dm.computeSweepCuts()
    part, srt = dm.downloadPartition(), orc.sorted()
    np.testing.assert_array_equal(part["nix"], srt["nix"])
    np.testing.assert_array_equal(part["prefix_edge_diff"], srt["prefix_edge_diff"])
    np.testing.assert_array_equal(part["prefix_volume"], srt["prefix_volume"])
    np.testing.assert_array_equal(part["offset_in_cluster"], srt["offset"])
    cuts, oc = dm.readSweepCuts(), orc.all_cuts()
    np.testing.assert_array_equal(cuts.clusterIds, oc["label"])
    np.testing.assert_array_equal(cuts.cuts["offset"], oc["offset"])
    np.testing.assert_array_equal(_bits(cuts.cuts["sparsity"]), _bits(oc["sparsity"]))
    if orc.n_active == 0:
        return False
    orc.cut_clusters()
    dm.cutClusters()
    np.testing.assert_array_equal(dm.downloadLabels(), orc.labels())
    np.testing.assert_array_equal(_bits(dm.readRandomWalkValues()), _bits(orc.potentials()))
    np.testing.assert_array_equal(dm.downloadDegrees(), orc.internal_degrees())
    np.testing.assert_array_equal(dm.downloadGraph()[1], orc.cols())
    assert dm.getNumClusters() == orc.n_clusters
    return orc.n_clusters > 0 and orc.n_active > 0


@pytest.mark.parametrize("name", sorted(SMALL))
def test_every_stage_of_every_round_bit_exact(name):
    g = SMALL[name]()
    dm, orc = _pair(g)
    for _ in range(1000):
        if not _check_round(dm, orc):
            break
    ids, k = orc.final_partition()
    fp = dm.getFinalPartition()
    np.testing.assert_array_equal(fp.clusterIds, ids)
    assert fp.numClusters == k
    assert dm.getNumCutEdges() == orc.num_cut_edges()


@pytest.mark.parametrize("name", ["sbm2k", "grid16", "rmat11", "path", "isolated"])
@pytest.mark.parametrize("driver", [P.DRIVER_STREAM, P.DRIVER_GRAPH])
def test_decomposition_end_to_end_bit_exact(name, driver):
    g = SMALL[name]()
    dm = P.CudaDeviceManager(driver=driver)
    dm.initialize(g)
    x0 = dm.readRandomWalkValues()
    rounds = dm.expanderDecomposition()
    orc = O.Oracle(g.offsets, g.cols, O.MODE_PXR)
    orc.set_potentials(x0.astype(np.float64))
    assert rounds == orc.decompose()
    np.testing.assert_array_equal(dm.downloadLabels(), orc.labels())
    ids, k = orc.final_partition()
    fp = dm.getFinalPartition()
    np.testing.assert_array_equal(fp.clusterIds, ids)
    assert fp.numClusters == k
    assert dm.getNumCutEdges() == orc.num_cut_edges()
    np.testing.assert_array_equal(dm.downloadGraph()[1], orc.cols())


def test_sbm16k_config1_end_to_end_bit_exact():
    """Planted partition n=16384, 16 blocks, degrees 12 / 0.5, seed 6582."""
    g = G.sbm_graph()
    dm = P.CudaDeviceManager()
    dm.initialize(g)
    x0 = dm.readRandomWalkValues()
    dm.expanderDecomposition()
    orc = O.Oracle(g.offsets, g.cols, O.MODE_PXR)
    orc.set_potentials(x0.astype(np.float64))
    orc.decompose()
    ids, k = orc.final_partition()
    fp = dm.getFinalPartition()
    np.testing.assert_array_equal(fp.clusterIds, ids)
    assert dm.getNumCutEdges() == orc.num_cut_edges()


def test_initial_potentials_match_oracle_within_4_ulps():
    g = G.grid3d(16)
    dm = P.CudaDeviceManager(seed=123)
    dm.initialize(g)
    x = dm.readRandomWalkValues()
    xo = O.initial_potentials(g.offsets, 123)
    assert np.all(np.abs(x.astype(np.float64) - xo) <= 4 * np.spacing(np.abs(xo)))


def test_repeated_walks_and_sweeps_without_cut():
    """Walk and sweep may be called repeatedly without a cut, as the
    reference's SweepCut test does (tests/cudaTest.cpp:141-166)."""
    g = G.sbm_graph(2048, 8, 10.0, 0.5, 7)
    dm, orc = _pair(g)
    for _ in range(6):
        orc.walk(); dm.iterateRandomWalk()
        orc.sweep(); dm.computeSweepCuts()
        np.testing.assert_array_equal(_bits(dm.readRandomWalkValues()), _bits(orc.potentials()))
        np.testing.assert_array_equal(_bits(dm.readSweepCuts().cuts["sparsity"]), _bits(orc.all_cuts()["sparsity"]))


def test_64bit_offsets_path():
    g = G.grid3d(12)
    g64 = G.CSRGraph(g.offsets.astype(np.uint64), g.cols, "grid12_64")
    a = P.CudaDeviceManager(); a.initialize(g); a.expanderDecomposition()
    b = P.CudaDeviceManager(); b.initialize(g64); b.expanderDecomposition()
    np.testing.assert_array_equal(a.getFinalPartition().clusterIds, b.getFinalPartition().clusterIds)


def test_invalid_input_is_rejected():
    dm = P.CudaDeviceManager()
    bad = G.CSRGraph(np.array([0, 2, 1], dtype=np.uint32), np.array([1, 0], dtype=np.uint32))
    with pytest.raises(P.PxrError):
        dm.initialize(bad)
    bad_col = G.CSRGraph(np.array([0, 1, 2], dtype=np.uint32), np.array([1, 7], dtype=np.uint32))
    with pytest.raises(P.PxrError):
        dm.initialize(bad_col)
    with pytest.raises(P.PxrError):
        P.CudaDeviceManager().iterateRandomWalk()


def test_round_cap_reports_iter_cap():
    g = G.grid3d(16)
    dm = P.CudaDeviceManager(max_rounds=3)
    dm.initialize(g)
    with pytest.raises(P.PxrError) as e:
        dm.expanderDecomposition()
    assert e.value.status == 3
