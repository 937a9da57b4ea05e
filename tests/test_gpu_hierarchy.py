"""Expander hierarchy on the GPU (parex_b200/hierarchy.py, pxr_contract): the
consumer the reference's drop-in hook computeExpanderDecomposition<true>
names (lib/algorithms/expander_hierarchy.h:91-101).

* pxr_contract equals a numpy restatement of ExpanderHierarchy::contract
  (:34-88): one vertex per cluster, one edge per cut edge (multi-edges kept,
  rows compared as sorted lists since the reference keeps its clusters' vertex
  order), cut sizes, and volumes (degrees at the first level, sums of the
  level below above it);
* a whole hierarchy ends in one vertex, and at every level the volumes add
  up to the input graph's volume and the cut sizes to twice the next level's
  edges.
"""
import numpy as np
import pytest
import torch

import parex_b200 as P
from parex_b200 import graphs as G, hierarchy as H

pytestmark = pytest.mark.gpu


def _restated_contract(offsets, cols, ids, k, level_vol=None):
    n = offsets.shape[0] - 1
    deg = np.diff(offsets.astype(np.int64))
    src = np.repeat(np.arange(n), deg)
    cut = ids[src] != ids[cols]
    a, b = ids[src][cut].astype(np.int64), ids[cols][cut].astype(np.int64)
    order = np.lexsort((b, a))
    out_cols = b[order]
    out_off = np.zeros(k + 1, dtype=np.int64)
    np.cumsum(np.bincount(a, minlength=k), out=out_off[1:])
    cut_sizes = np.bincount(a, minlength=k)
    vols = np.bincount(ids, weights=deg if level_vol is None else level_vol, minlength=k).astype(np.int64)
    return out_off, out_cols, cut_sizes, vols


def test_contract_matches_the_restated_contraction():
    g = G.sbm_graph()
    dm = P.CudaDeviceManager()
    dm.initialize(g)
    dm.expanderDecomposition()
    fp = dm.getFinalPartition()
    off = torch.from_numpy(g.offsets.view(np.int32)).cuda()
    cols = torch.from_numpy(g.cols.view(np.int32)).cuda()
    ids = torch.from_numpy(fp.clusterIds).cuda()
    noff, ncol, m, cut, vol = H.contract(off, cols, ids, fp.numClusters)
    want_off, want_cols, want_cut, want_vol = _restated_contract(g.offsets, g.cols, fp.clusterIds, fp.numClusters)
    np.testing.assert_array_equal(noff.cpu().numpy(), want_off)
    np.testing.assert_array_equal(ncol.cpu().numpy(), want_cols)
    np.testing.assert_array_equal(cut.cpu().numpy(), want_cut)
    np.testing.assert_array_equal(vol.cpu().numpy(), want_vol)
    assert m == dm.countCutEdges()
    # a second level: volumes are sums of the level below
    k2 = max(1, fp.numClusters // 7)
    ids2 = (np.arange(fp.numClusters) % k2).astype(np.int32)
    o2, c2, m2, cut2, vol2 = H.contract(noff, ncol, torch.from_numpy(ids2).cuda(), k2, vol)
    w_off, w_cols, w_cut, w_vol = _restated_contract(want_off, want_cols.astype(np.uint32), ids2, k2, want_vol)
    np.testing.assert_array_equal(o2.cpu().numpy(), w_off)
    np.testing.assert_array_equal(c2.cpu().numpy(), w_cols)
    np.testing.assert_array_equal(cut2.cpu().numpy(), w_cut)
    np.testing.assert_array_equal(vol2.cpu().numpy(), w_vol)


@pytest.mark.parametrize("name", ["sbm16k", "grid16"])
def test_hierarchy_reaches_one_vertex(name):
    g = {"sbm16k": lambda: G.sbm_graph(), "grid16": lambda: G.grid3d(16)}[name]()
    levels = H.build(torch.from_numpy(g.offsets.view(np.int32)), torch.from_numpy(g.cols.view(np.int32)))
    assert levels and levels[-1].clusters == 1
    total = 2 * g.m
    n = g.n
    for i, lvl in enumerate(levels):
        assert lvl.n == n and lvl.parents.shape[0] == n
        assert int(lvl.volumes.sum()) == total
        assert int(lvl.cut_sizes.sum()) == 2 * lvl.cut_edges
        if i + 1 < len(levels):
            assert levels[i + 1].m == lvl.cut_edges
        n = lvl.clusters


def _ncut(g, labels):
    src = np.repeat(np.arange(g.n), np.diff(g.offsets.astype(np.int64)))
    deg = np.diff(g.offsets.astype(np.int64))
    k = int(labels.max()) + 1
    cut = np.bincount(labels[src], weights=(labels[src] != labels[g.cols]).astype(np.float64), minlength=k)
    vol = np.bincount(labels, weights=deg, minlength=k)
    keep = vol > 0
    return float(np.sum(cut[keep] / vol[keep]))


def test_normalized_cut_finds_the_planted_blocks():
    from parex_b200.normalized_cut import NormalizedCut
    g = G.sbm_graph()            # 16 planted blocks
    levels = H.build(torch.from_numpy(g.offsets.view(np.int32)), torch.from_numpy(g.cols.view(np.int32)))
    labels = NormalizedCut(levels, g.n).compute(16)
    assert labels.min() >= 0 and labels.max() <= 16
    rng = np.random.default_rng(0)
    random = rng.integers(0, int(labels.max()) + 1, g.n)
    assert _ncut(g, labels) < 0.5 * _ncut(g, random)
