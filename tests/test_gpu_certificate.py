"""Certificates of the GPU decomposition, plain and learned.

* The certificate record (pxr_download_certificates) equals the oracle's
  bit for bit after a plain decomposition from the same potentials.
* Every output cluster passes the end-to-end check of
  parex_b200/certificate.py: certified by the keep test
  (cuda/devPartition.h:173-184), no sweep prefix below sc where the cluster
  was certified whole (cuda/devSweepCut.h:321-331), connected, internal
  degrees equal to induced degrees - under the plain form and under the
  learned schedule with the shipped model.
* pxr_count_cut_edges equals the host recount over the final ids
  (main.cpp:54-60), and downloadGraph shows disabled slots as INVALID_EDGE.
"""
import numpy as np
import pytest

import parex_b200 as P
from oracle import oracle as O
from parex_b200 import _lib, certificate as CERT, graphs as G, learn

pytestmark = pytest.mark.gpu

SC, RW = 0.3, 1e-4

GRAPHS = {
    "sbm16k": lambda: G.sbm_graph(),
    "grid32": lambda: G.grid3d(32),
    "rmat14": lambda: G.rmat(14, 16, seed=3),
    "regular": lambda: G.random_regular(1 << 14, 8, seed=2),
    "path": lambda: G.csr_from_edges(np.arange(999, dtype=np.uint32), np.arange(1, 1000, dtype=np.uint32), 1000),
}


def _recount(g, ids):
    src = np.repeat(np.arange(g.n), np.diff(g.offsets.astype(np.int64)))
    return int(np.count_nonzero(ids[src] != ids[g.cols]) // 2)


def _check(g, dm, fp):
    return CERT.check(g.offsets, g.cols, fp.clusterIds, dm.readRandomWalkValues(), dm.downloadCertificates(),
                      SC, RW, device="cuda", degrees=dm.downloadDegrees())


@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_plain_certificates_match_oracle_and_check(name):
    g = GRAPHS[name]()
    dm = P.CudaDeviceManager()
    dm.initialize(g)
    x0 = dm.readRandomWalkValues()
    dm.expanderDecomposition()
    orc = O.Oracle(g.offsets, g.cols, O.MODE_PXR, SC, RW)
    orc.set_potentials(x0.astype(np.float64))
    orc.decompose()
    np.testing.assert_array_equal(dm.downloadCertificates(), orc.certificates())
    fp = dm.getFinalPartition()
    rep = _check(g, dm, fp)
    assert rep["ok"], rep
    assert dm.countCutEdges() == rep["cut_edges"] == _recount(g, fp.clusterIds)
    # the mutated graph as the reference returns it
    np.testing.assert_array_equal(dm.downloadGraph()[1], orc.cols())


@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_learned_certificates_check(name):
    g = GRAPHS[name]()
    model = learn.Model.load()
    dm = P.CudaDeviceManager()
    dm.set_schedule(_lib.SCHEDULE_LEARNED, model.weights, model.norm, **learn.SHIPPED_SCHEDULE)
    dm.initialize(g)
    dm.expanderDecomposition()
    fp = dm.getFinalPartition()
    rep = _check(g, dm, fp)
    assert rep["ok"], rep
    assert dm.countCutEdges() == _recount(g, fp.clusterIds)


def test_count_cut_edges_on_device_graph_and_64bit_offsets():
    g = G.sbm_graph(4096, 8, 10.0, 0.5, 5)
    dm = P.CudaDeviceManager()
    dm.initialize((g.offsets.astype(np.uint64), g.cols))
    dm.expanderDecomposition()
    assert dm.countCutEdges() == _recount(g, dm.getFinalPartition().clusterIds)


def test_count_cut_edges_refuses_unknown_neighbours():
    g = G.grid3d(8)
    dm = P.CudaDeviceManager()
    dm.initialize(g)
    cols = g.cols.copy()
    cols[0] = 0xFFFFFFFF    # a disabled slot loaded without its neighbour
    dm.set_state(np.zeros(g.n, np.int32), np.arange(g.n, dtype=np.uint32), np.zeros(g.n), np.diff(
        g.offsets).astype(np.uint32), cols, 1, 0)
    with pytest.raises(_lib.PxrError):
        dm.countCutEdges()
