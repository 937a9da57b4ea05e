"""Row plans and the autotuner (pxr_get_row_plan / pxr_set_row_plan).

The plan (lanes per light row, warp- and CTA-per-row bins) changes speed
only: decompositions under the tuned plan and under forced plans that put
rows in every bin must agree bit for bit.  The tuner's choice is cached per
degree histogram.
"""
import numpy as np
import pytest

import parex_b200 as P
from parex_b200 import graphs as G

pytestmark = pytest.mark.gpu


def _edges_graph(n, edges):
    e = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
    return G.csr_from_edges(e[:, 0], e[:, 1], n)


GRAPHS = {
    "rmat13": lambda: G.rmat(13, 16, seed=4),
    "grid12": lambda: G.grid3d(12),
    "star": lambda: _edges_graph(3000, [(0, i) for i in range(1, 3000)] + [(i, i + 1) for i in range(1, 2999)]),
    "sbm2k": lambda: G.sbm_graph(2048, 8, 10.0, 0.5, 7),
}
PLANS = [(1, 16, 1024), (4, 32, 64), (32, 128, 16384), (8, 4, 8), (16, 1, 1)]


def _run(g, plan=None, driver=P.DRIVER_GRAPH):
    dm = P.CudaDeviceManager(driver=driver)
    if plan is not None:
        dm.set_row_plan(*plan)
    dm.initialize(g)
    dm.expanderDecomposition()
    fp = dm.getFinalPartition()
    return fp.clusterIds, dm.getNumCutEdges(), dm.readRandomWalkValues(), dm.row_plan()


@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_results_do_not_depend_on_the_plan(name):
    g = GRAPHS[name]()
    ids, cut, x, rp = _run(g)
    assert rp["source"] in (1, 2)
    assert rp["lanes_per_row"] in (1, 4, 8, 16, 32)
    for plan in PLANS:
        ids2, cut2, x2, rp2 = _run(g, plan, driver=P.DRIVER_STREAM if plan[0] == 8 else P.DRIVER_GRAPH)
        assert rp2["source"] == 3 and rp2["lanes_per_row"] == plan[0]
        np.testing.assert_array_equal(ids, ids2)
        assert cut == cut2
        np.testing.assert_array_equal(x.view(np.uint32), x2.view(np.uint32))
    # a plan with every long row in the CTA bin and one with every row in the warp bin
    deg = np.diff(g.offsets.astype(np.int64))
    if deg.max() > 1:
        _, _, _, rp3 = _run(g, (4, 1, 1))
        assert rp3["heavy_rows"] == int(np.count_nonzero(deg > 1)) and rp3["wide_rows"] == 0
        _, _, _, rp4 = _run(g, (4, 1, 1 << 30))
        assert rp4["wide_rows"] == int(np.count_nonzero(deg > 1)) and rp4["heavy_rows"] == 0


def test_tuned_plan_is_cached():
    g = G.rmat(12, 16, seed=9)
    a = P.CudaDeviceManager()
    a.initialize(g)
    first = a.row_plan()
    b = P.CudaDeviceManager()
    b.initialize(g)
    second = b.row_plan()
    assert second["source"] == 2
    assert first["source"] in (1, 2)
    for k in ("lanes_per_row", "light_max", "wide_max", "wide_rows", "heavy_rows"):
        assert first[k] == second[k]
    h = P.CudaDeviceManager(tune=P.TUNE_HEURISTIC)
    h.initialize(g)
    assert h.row_plan()["source"] == 0


def test_forced_plan_validation_and_reset():
    g = G.grid3d(8)
    dm = P.CudaDeviceManager()
    with pytest.raises(P.PxrError):
        dm.set_row_plan(3, 64, 4096)
    with pytest.raises(P.PxrError):
        dm.set_row_plan(4, 64, 32)
    dm.initialize(g)
    dm.set_row_plan(16, 8, 16)
    assert dm.row_plan()["source"] == 3
    dm.expanderDecomposition()
    dm.set_row_plan()
    assert dm.row_plan()["source"] in (1, 2)


@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_components_schedules_agree(name):
    """Plain and sampled union-find give the same components, so the same
    decomposition, in both drivers (the sampled schedule skips the rows of
    each label's representative set: a different order of joins only)."""
    g = GRAPHS[name]()
    out = []
    for comp in (P.COMPONENTS_PLAIN, P.COMPONENTS_SAMPLED):
        for driver in (P.DRIVER_GRAPH, P.DRIVER_STREAM):
            dm = P.CudaDeviceManager(driver=driver, components=comp)
            dm.initialize(g)
            dm.expanderDecomposition()
            out.append((dm.getFinalPartition().clusterIds, dm.getNumCutEdges(), dm.downloadLabels()))
            dm.close()
    for ids, cut, lab in out[1:]:
        np.testing.assert_array_equal(ids, out[0][0])
        assert cut == out[0][1]
        np.testing.assert_array_equal(lab, out[0][2])


# ---------------------------------------------------------------------------
# sort plans (pxr_get_sort_plan / pxr_set_sort_plan): keys per thread and CTAs
# per SM of the sweep's radix sort change speed only


@pytest.mark.parametrize("name", ["rmat13", "grid12"])
@pytest.mark.parametrize("driver", [P.DRIVER_GRAPH, P.DRIVER_STREAM])
def test_results_do_not_depend_on_the_sort_plan(name, driver):
    g = GRAPHS[name]()
    runs = []
    for plan in (0, 1, 2):
        dm = P.CudaDeviceManager(driver=driver)
        dm.set_sort_plan(plan)
        dm.initialize(g)
        dm.expanderDecomposition()
        sp = dm.sort_plan()
        assert sp["plan"] == plan and sp["source"] == 3
        assert (sp["items_per_thread"], sp["ctas_per_sm"]) == [(16, 2), (12, 3), (8, 4)][plan]
        runs.append((dm.getFinalPartition().clusterIds, dm.downloadLabels(), dm.readRandomWalkValues()))
    for ids, labels, x in runs[1:]:
        np.testing.assert_array_equal(ids, runs[0][0])
        np.testing.assert_array_equal(labels, runs[0][1])
        np.testing.assert_array_equal(x.view(np.uint32), runs[0][2].view(np.uint32))


def test_sort_plan_is_tuned_and_cached():
    g = G.grid3d(48)     # 110,592 vertices: above the tuning threshold
    a = P.CudaDeviceManager()
    a.initialize(g)
    first = a.sort_plan()
    assert first["source"] in (1, 2) and first["plan"] in (0, 1, 2)
    assert all(t > 0 for t in first["sort_us"])
    assert first["plan"] == int(np.argmin(first["sort_us"]))
    b = P.CudaDeviceManager()
    b.initialize(g)
    assert b.sort_plan()["source"] == 2 and b.sort_plan()["plan"] == first["plan"]
    # the probe sorts are not counted as sweep traffic
    assert b.stats()["sort_items"] == 0
    with pytest.raises(Exception):
        b.set_sort_plan(3)
