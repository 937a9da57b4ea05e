"""Normalized cut over an expander hierarchy (parex_b200/normalized_cut.py,
the greedy of lib/algorithms/normalized_cut.h:109-141), on the CPU with a
hand-built two-level hierarchy: two triangles joined by one edge, each
triangle a cluster.  One split must separate the triangles (the cheapest
normalized cut), and the bookkeeping must move the split node's volume and
cut up to the root."""
import numpy as np

from parex_b200.hierarchy import Level
from parex_b200.normalized_cut import NormalizedCut


def _two_triangles():
    # graph: 0-1-2 triangle, 3-4-5 triangle, edge 2-3; volume 14, cut 1 between the triangles
    lvl0 = Level(n=6, m=7, clusters=2, cut_edges=1, sc_threshold=0.3,
                 parents=np.array([0, 0, 0, 1, 1, 1]), volumes=np.array([7, 7]), cut_sizes=np.array([1, 1]))
    lvl1 = Level(n=2, m=1, clusters=1, cut_edges=0, sc_threshold=0.3,
                 parents=np.array([0, 0]), volumes=np.array([14]), cut_sizes=np.array([0]))
    return [lvl0, lvl1]


def test_one_split_separates_the_triangles():
    nc = NormalizedCut(_two_triangles(), 6)
    labels = nc.compute(1)
    # labels come from the last search, which ran with the root alone
    assert np.array_equal(labels, np.zeros(6))
    assert (0, 0) in nc.roots or (0, 1) in nc.roots
    # the split node's volume left the root, its cut was added there
    assert nc.volumes[1][0] == 7 and nc.cuts[1][0] == 1
    labels = nc.compute(2)
    assert len(set(labels[:3])) == 1 and len(set(labels[3:])) == 1


def test_penalty_is_float32_normalized_cut_change():
    nc = NormalizedCut(_two_triangles(), 6)
    pen = nc._edge_penalty(0, 0, 0, 14)
    assert pen == np.float32(1 / 7) + np.float32(1 / 7)
