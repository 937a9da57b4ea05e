"""The benchmark workload at full size: 3D 7-point grid 128^3
(n = 2,097,152, m = 6,242,304), seed 6582, sc 0.3, rw 1e-4.

* bit-exact against the oracle (ORC_MODE_PXR) end to end: labels, final
  partition, disabled slots, round count;
* deterministic: two runs give identical labels and potentials;
* band: cluster count and device cut edges (m - valid/2) within 1 %, and the
  recounted cut (edges whose endpoints carry different final ids, as
  main.cpp:54-60 counts them) within 2 % of the reference binary's figures on
  the same graph and seed.
"""
import numpy as np
import pytest

import parex_b200 as P
from parex_b200 import graphs as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# the reference binary on B200 (oracle/_ref/ref_gpu decomp, seed 6582)
REF_GRID128 = {"num_clusters_fp": 807627, "cut_edges_recount": 4666329, "cut_edges_device": 3727842,
               "iterations_printed": 50}


@pytest.fixture(scope="module")
def grid128():
    return G.grid3d(128)


@pytest.fixture(scope="module")
def run128(grid128):
    dm = P.CudaDeviceManager()
    dm.initialize(grid128)
    x0 = dm.readRandomWalkValues()
    rounds = dm.expanderDecomposition()
    return dm, x0, rounds


def test_grid128_bit_exact_against_oracle(grid128, run128):
    dm, x0, rounds = run128
    orc = O.Oracle(grid128.offsets, grid128.cols, O.MODE_PXR)
    orc.set_potentials(x0.astype(np.float64))
    assert orc.decompose() == rounds
    np.testing.assert_array_equal(dm.downloadLabels(), orc.labels())
    np.testing.assert_array_equal(dm.downloadGraph()[1], orc.cols())
    ids, k = orc.final_partition()
    fp = dm.getFinalPartition()
    assert fp.numClusters == k
    np.testing.assert_array_equal(fp.clusterIds, ids)


def test_grid128_deterministic(grid128, run128):
    dm, x0, _ = run128
    again = P.CudaDeviceManager(driver=P.DRIVER_STREAM)
    again.initialize(grid128)
    again.expanderDecomposition()
    np.testing.assert_array_equal(again.downloadLabels(), dm.downloadLabels())
    np.testing.assert_array_equal(again.readRandomWalkValues().view(np.uint32),
                                  dm.readRandomWalkValues().view(np.uint32))


def test_grid128_band_against_reference(grid128, run128):
    dm, _, rounds = run128
    fp = dm.getFinalPartition()
    src = np.repeat(np.arange(grid128.n), np.diff(grid128.offsets.astype(np.int64)))
    ids = fp.clusterIds
    recount = int(np.sum(ids[src] != ids[grid128.cols]) // 2)
    device = dm.getNumCutEdges()
    assert abs(fp.numClusters - REF_GRID128["num_clusters_fp"]) <= 0.01 * REF_GRID128["num_clusters_fp"]
    assert abs(device - REF_GRID128["cut_edges_device"]) <= 0.01 * REF_GRID128["cut_edges_device"]
    assert abs(recount - REF_GRID128["cut_edges_recount"]) <= 0.02 * REF_GRID128["cut_edges_recount"]
    assert abs(rounds - REF_GRID128["iterations_printed"]) <= 5
