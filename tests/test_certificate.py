"""The end-to-end certificate check (parex_b200/certificate.py) on the CPU.

* Every cluster of the oracle's decomposition (plain rounds, and rounds under
  a sweep schedule that skips clusters) passes: certified by the keep test
  (cuda/devPartition.h:173-184), no sweep prefix below sc for clusters
  certified whole (cuda/devSweepCut.h:321-331), connected through its own
  edges (tests/clusterTest.cpp:11-40).
* Mistakes planted in the oracle's output are caught: a potential spread
  above the threshold, a sparse cut inside a cluster certified whole, two
  certified clusters merged, a vertex left uncertified.
* The recounted cut edges equal a direct count over the final ids.
"""
import numpy as np
import pytest

from oracle import oracle as O
from parex_b200 import certificate as CERT
from parex_b200 import graphs as G

SC, RW = 0.3, 1e-4

GRAPHS = {
    "sbm2k": lambda: G.sbm_graph(2048, 8, 10.0, 0.5, 7),
    "sbm16k": lambda: G.sbm_graph(),
    "grid16": lambda: G.grid3d(16),
    "rmat12": lambda: G.rmat(12, 16, seed=3),
    "regular": lambda: G.random_regular(4096, 8, seed=2),
}


def _decompose(g, seed=6582):
    x0 = O.initial_potentials(g.offsets, seed)
    orc = O.Oracle(g.offsets, g.cols, O.MODE_PXR, SC, RW)
    orc.set_potentials(x0.astype(np.float64))
    orc.decompose()
    return orc


def _check(g, orc, ids=None, x=None, cert=None):
    if ids is None:
        ids, _ = orc.final_partition()
    return CERT.check(g.offsets, g.cols, ids, orc.potentials().astype(np.float32) if x is None else x,
                      orc.certificates() if cert is None else cert, SC, RW, degrees=orc.internal_degrees())


def _recount(g, ids):
    src = np.repeat(np.arange(g.n), np.diff(g.offsets.astype(np.int64)))
    return int(np.count_nonzero(ids[src] != ids[g.cols]) // 2)


@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_oracle_decomposition_is_certified(name):
    g = GRAPHS[name]()
    orc = _decompose(g)
    ids, k = orc.final_partition()
    rep = _check(g, orc)
    assert rep["ok"], rep
    assert rep["uncertified_vertices"] == 0
    assert rep["clusters"] >= k     # final ids may merge clusters that reused a label
    assert rep["sweep_checked"] > 0
    assert rep["cut_edges"] == _recount(g, ids)


def test_scheduled_rounds_are_certified():
    """Skipping sweeps (a random schedule) never certifies a cluster without
    the keep test, nor leaves a sparse cut inside a cluster certified whole."""
    g = G.sbm_graph(4096, 16, 10.0, 0.5, 11)
    x0 = O.initial_potentials(g.offsets, 6582)
    orc = O.Oracle(g.offsets, g.cols, O.MODE_PXR, SC, RW)
    orc.set_potentials(x0.astype(np.float64))
    rng = np.random.default_rng(4)
    rounds = 0
    while orc.n_clusters > 0 and orc.n_active > 0 and rounds < 5000:
        due = (rng.random(orc.n_clusters) < 0.4).astype(np.uint8)
        orc.scheduled_round(due)
        rounds += 1
    assert orc.n_active == 0 or orc.n_clusters == 0
    rep = _check(g, orc)
    assert rep["ok"], rep


def test_planted_spread_is_caught():
    g = GRAPHS["sbm2k"]()
    orc = _decompose(g)
    ids, _ = orc.final_partition()
    cert = orc.certificates()
    x = orc.potentials().astype(np.float32)
    # a certified cluster of at least two vertices: raise one potential
    key = ids.astype(np.int64) * (int(cert.max() & 0x7FFFFFFF) + 1) + (cert & 0x7FFFFFFF)
    vals, counts = np.unique(key, return_counts=True)
    v = int(np.flatnonzero(key == vals[np.argmax(counts)])[0])
    x[v] += np.float32(4 * RW)
    rep = _check(g, orc, x=x)
    assert not rep["ok"] and rep["threshold_violations"] == 1


def test_planted_sparse_cut_is_caught():
    """Two 8-cliques joined by one edge, reported as one cluster certified
    whole with flat potentials: the keep test passes, the sweep does not."""
    k = 8
    edges = [(a, b) for a in range(k) for b in range(a + 1, k)]
    edges += [(k + a, k + b) for a in range(k) for b in range(a + 1, k)]
    edges.append((0, k))
    e = np.array(edges, dtype=np.uint32)
    g = G.csr_from_edges(e[:, 0], e[:, 1], 2 * k)
    ids = np.zeros(2 * k, dtype=np.int32)
    x = np.concatenate([np.zeros(k), np.full(k, 1e-5)]).astype(np.float32)
    cert = np.ones(2 * k, dtype=np.uint32)
    rep = CERT.check(g.offsets, g.cols, ids, x, cert, SC, RW)
    assert rep["threshold_violations"] == 0
    assert rep["sweep_violations"] == 1 and not rep["ok"]
    assert rep["min_sweep_sparsity"] == pytest.approx(1 / 57, rel=1e-6)
    # the same set certified as a piece of a cut cluster: only the keep test applies
    rep = CERT.check(g.offsets, g.cols, ids, x, cert | np.uint32(CERT.CUT_BIT), SC, RW)
    assert rep["ok"] and rep["sweep_checked"] == 0


def test_planted_merge_and_uncertified_vertex_are_caught():
    g = GRAPHS["grid16"]()
    orc = _decompose(g)
    ids, _ = orc.final_partition()
    cert = orc.certificates()
    # give two non-adjacent certified clusters one id and one round
    far = [0, g.n - 1]
    ids2 = ids.copy()
    cert2 = cert.copy()
    a, b = ids[far[0]], ids[far[1]]
    sel_b = ids == b
    ids2[sel_b] = a
    cert2[ids2 == a] = cert[far[0]]
    rep = _check(g, orc, ids=ids2, cert=cert2)
    assert not rep["ok"] and rep["disconnected"] >= 1
    cert3 = cert.copy()
    cert3[5] = 0
    rep = _check(g, orc, cert=cert3)
    assert not rep["ok"] and rep["uncertified_vertices"] == 1
