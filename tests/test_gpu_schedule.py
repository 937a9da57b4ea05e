"""The learned sweep schedule on the GPU.

* Trace mode leaves the plain decomposition unchanged and its per-cluster
  features match the oracle's restatement.
* Scheduled rounds match the oracle's scheduled round (orc_scheduled_round)
  bit for bit, given the schedule the product chose (read from the trace
  records): every cut is chosen and scored by the exact sweep.
* The audit mode gives the same partition as the learned mode and counts
  the skipped sweeps that would have cut.
"""
import numpy as np
import pytest

import parex_b200 as P
from oracle import mlp as M
from oracle import oracle as O
from parex_b200 import _lib, graphs as G, learn

pytestmark = pytest.mark.gpu

GRAPHS = {
    "sbm2k": lambda: G.sbm_graph(2048, 8, 10.0, 0.5, 7),
    "grid16": lambda: G.grid3d(16),
    "rmat11": lambda: G.rmat(11, 16, seed=3),
}


def _random_model(seed=0):
    """A random network whose predictions spread over 0..4 skipped rounds."""
    rng = np.random.default_rng(seed)
    w = learn.init_master(seed)
    w[M.OFF_B3] = 1.2
    norm = np.concatenate([np.zeros(16), rng.uniform(0.1, 0.6, 16)]).astype(np.float32)
    return learn.Model(learn.to_bf16_bits(w), norm)


def _bits(x):
    return np.asarray(x, dtype=np.float32).view(np.uint32)


@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_trace_keeps_plain_result_and_features(name):
    g = GRAPHS[name]()
    a = P.CudaDeviceManager(driver=P.DRIVER_STREAM)
    a.initialize(g)
    a.expanderDecomposition()
    b = P.CudaDeviceManager(driver=P.DRIVER_STREAM)
    b.set_schedule(_lib.SCHEDULE_PLAIN, trace=True)
    b.initialize(g)
    checked = 0
    while b.getNumClusters() > 0:
        b.iterateRandomWalk()
        b.computeSweepCuts()
        b.cutClusters()
        rec = b.cluster_records()
        if rec.shape[0]:
            f = M.features(rec, 1e-4, 0.3)
            np.testing.assert_allclose(rec["features"], f, rtol=2e-5, atol=2e-5)
            assert np.all(rec["origin"] != learn.ORIGIN_CARRIED)
            checked += rec.shape[0]
    assert checked > 0
    np.testing.assert_array_equal(a.getFinalPartition().clusterIds, b.getFinalPartition().clusterIds)


@pytest.mark.parametrize("gate,period", [(0.0, 0), (0.02, 0), (0.0, 3), (0.02, 3)])
@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_scheduled_rounds_match_oracle(name, gate, period):
    g = GRAPHS[name]()
    model = _random_model(1)
    dm = P.CudaDeviceManager(driver=P.DRIVER_STREAM)
    dm.set_schedule(_lib.SCHEDULE_LEARNED, model.weights, model.norm, safety=1.0, max_skip=4, trace=True,
                    cut_gate=gate, due_period=period)
    dm.initialize(g)
    orc = O.Oracle(g.offsets, g.cols, O.MODE_PXR)
    orc.set_potentials(dm.readRandomWalkValues().astype(np.float64))
    due = np.ones(1, dtype=np.uint8)
    skipped = 0
    gated_rounds = 0
    for _ in range(500):
        if dm.getNumClusters() == 0:
            break
        assert orc.n_clusters == dm.getNumClusters()
        k_round = np.float32(dm.getNumClusters())
        a_round = int(dm.stats()["active_vertices"])
        orc.scheduled_round(due)
        dm.iterateRandomWalk()
        dm.computeSweepCuts()
        cut = np.float32(dm.stats()["clusters_with_cut"])   # clusters this round's sweep cuts
        dm.cutClusters()
        np.testing.assert_array_equal(dm.downloadLabels(), orc.labels())
        np.testing.assert_array_equal(_bits(dm.readRandomWalkValues()), _bits(orc.potentials()))
        np.testing.assert_array_equal(dm.downloadDegrees(), orc.internal_degrees())
        np.testing.assert_array_equal(dm.downloadGraph()[1], orc.cols())
        rec = dm.cluster_records()
        # the cut gate: a round that cut more than gate x its clusters is followed by a full sweep
        gated = gate > 0 and cut > np.float32(gate) * k_round
        if gated:
            assert np.all(rec["skip"] == 0)
            gated_rounds += 1
        # the due period: outside its rounds no small cluster is due next round
        held_round = period > 1 and not gated and dm.stats()["rounds"] % period != 0
        held = held_round & (rec["size"].astype(np.uint64) * 1024 < a_round)
        assert np.all(rec["skip"][held] >= 1)
        # the product's predictions are the oracle network's on the same features
        sw = rec["origin"] == learn.ORIGIN_SWEPT
        if np.any(sw):
            y, _ = M.forward(model.weights, model.norm, rec["features"][sw])
            np.testing.assert_array_equal(_bits(rec["prediction"][sw]), _bits(y))
            r = np.exp2(np.minimum(y.astype(np.float64), 16.0)) - 1.0
            clear = np.abs(r - np.round(r)) > 1e-4          # away from a rounding boundary of floor()
            want = np.zeros(int(np.count_nonzero(sw)), dtype=np.int64) if gated else M.skip_from_prediction(y, 1.0, 4)
            want = np.where(held[sw], np.maximum(want, 1), want)
            np.testing.assert_array_equal(rec["skip"][sw][clear], want[clear])
        due = (rec["skip"] == 0).astype(np.uint8)
        skipped += int(np.count_nonzero(rec["skip"]))
    assert dm.getNumClusters() == 0
    assert skipped > 0, "the random schedule should skip some sweeps"
    if gate and name != "rmat11":   # the R-MAT graph's sweeps rarely cut: its rounds stay below the gate
        assert gated_rounds > 0, "some round should cut more than the gate"
    ids, k = orc.final_partition()
    fp = dm.getFinalPartition()
    np.testing.assert_array_equal(fp.clusterIds, ids)
    assert fp.numClusters == k


@pytest.mark.parametrize("driver", [P.DRIVER_GRAPH, P.DRIVER_STREAM])
def test_audit_mode_same_partition(driver):
    g = G.grid3d(24)
    model = _random_model(2)
    res = {}
    for mode in (_lib.SCHEDULE_LEARNED, _lib.SCHEDULE_AUDIT):
        dm = P.CudaDeviceManager(driver=driver)
        dm.set_schedule(mode, model.weights, model.norm, safety=1.0, max_skip=4)
        dm.initialize(g)
        dm.expanderDecomposition()
        res[mode] = (dm.getFinalPartition().clusterIds, dm.stats())
    np.testing.assert_array_equal(res[1][0], res[2][0])
    assert res[1][1]["skipped_sweeps"] == res[2][1]["skipped_sweeps"] > 0
    assert res[2][1]["false_stops"] <= res[2][1]["skipped_sweeps"]
    assert res[1][1]["swept_items"] < res[2][1]["swept_items"]


def test_graph_and_stream_drivers_agree_in_learned_mode():
    g = G.sbm_graph(4096, 16, 12.0, 0.5, 5)
    model = _random_model(3)
    ids = []
    for driver in (P.DRIVER_GRAPH, P.DRIVER_STREAM):
        dm = P.CudaDeviceManager(driver=driver)
        dm.set_schedule(_lib.SCHEDULE_LEARNED, model.weights, model.norm, safety=1.0, max_skip=4)
        dm.initialize(g)
        dm.expanderDecomposition()
        ids.append(dm.getFinalPartition().clusterIds)
    np.testing.assert_array_equal(ids[0], ids[1])
