"""Parity at the full size of the benchmark's configurations (bit-exact
against the oracle in the product's arithmetic, ORC_MODE_PXR), with every
output cluster certified (parex_b200/certificate.py):

* R-MAT scale 22, edge factor 16 (a,b,c) = (.57,.19,.19), graph seed 1, built
  on the device (the batched-form configuration's graph);
* the random 8-regular graph on 2^22 vertices (the no-split case of the
  learned configuration), plain and under the learned schedule with the
  shipped model (the oracle replays the product's schedule round by round);
* 32 instances of the 512-instance planted-partition batch, stratified by
  size and including the largest, decomposed as one batch.

Each compares labels, final partition, certificate record and round count
with the oracle started from the product's own initial potentials.
"""
import numpy as np
import pytest

import parex_b200 as P
from oracle import oracle as O
from parex_b200 import _lib, certificate as CERT, gpu_build as B, graphs as G, learn

pytestmark = pytest.mark.gpu

SC, RW = 0.3, 1e-4


def _host(off_d, cols_d):
    off = off_d.cpu().numpy()
    off = off.view(np.uint64) if off.dtype == np.int64 else off.view(np.uint32)
    return off, cols_d.cpu().numpy().view(np.uint32)


def _certified(off, cols, dm, fp):
    rep = CERT.check(off, cols, fp.clusterIds, dm.readRandomWalkValues(), dm.downloadCertificates(), SC, RW,
                     device="cuda", degrees=dm.downloadDegrees())
    assert rep["ok"], rep
    return rep


def _plain_against_oracle(off, cols, dm, rounds, orc):
    assert orc.decompose() == rounds
    np.testing.assert_array_equal(dm.downloadLabels(), orc.labels())
    ids, k = orc.final_partition()
    fp = dm.getFinalPartition()
    assert fp.numClusters == k
    np.testing.assert_array_equal(fp.clusterIds, ids)
    np.testing.assert_array_equal(dm.downloadCertificates(), orc.certificates())
    _certified(off, cols, dm, fp)
    src = np.repeat(np.arange(off.shape[0] - 1), np.diff(off.astype(np.int64)))
    assert dm.countCutEdges() == int(np.count_nonzero(ids[src] != ids[cols]) // 2)


def test_rmat22_plain_bit_exact():
    off_d, cols_d, n, m = B.rmat(22, 16, seed=1)
    off, cols = _host(off_d, cols_d)
    dm = P.CudaDeviceManager()
    dm.initialize_device(n, m, off_d.data_ptr(), False, cols_d.data_ptr())
    x0 = dm.readRandomWalkValues()
    rounds = dm.expanderDecomposition()
    orc = O.Oracle(off, cols, O.MODE_PXR, SC, RW)
    orc.set_potentials(x0.astype(np.float64))
    _plain_against_oracle(off, cols, dm, rounds, orc)


@pytest.fixture(scope="module")
def regular22():
    return G.random_regular(1 << 22, 8, seed=1)


def test_regular22_plain_bit_exact(regular22):
    g = regular22
    dm = P.CudaDeviceManager()
    dm.initialize(g)
    x0 = dm.readRandomWalkValues()
    rounds = dm.expanderDecomposition()
    orc = O.Oracle(g.offsets, g.cols, O.MODE_PXR, SC, RW)
    orc.set_potentials(x0.astype(np.float64))
    _plain_against_oracle(g.offsets, g.cols, dm, rounds, orc)


def test_regular22_learned_shipped_model_bit_exact(regular22):
    """The shipped model's schedule, replayed by the oracle: every round's
    due set is the product's, and the end state is identical."""
    g = regular22
    model = learn.Model.load()
    dm = P.CudaDeviceManager(driver=P.DRIVER_STREAM)
    dm.set_schedule(_lib.SCHEDULE_LEARNED, model.weights, model.norm, trace=True, **learn.SHIPPED_SCHEDULE)
    dm.initialize(g)
    orc = O.Oracle(g.offsets, g.cols, O.MODE_PXR, SC, RW)
    orc.set_potentials(dm.readRandomWalkValues().astype(np.float64))
    due = np.ones(1, dtype=np.uint8)
    skipped = rounds = 0
    while dm.getNumClusters() > 0 and rounds < 2000:
        assert orc.n_clusters == dm.getNumClusters()
        orc.scheduled_round(due)
        dm.iterateRandomWalk()
        dm.computeSweepCuts()
        dm.cutClusters()
        rec = dm.cluster_records()
        due = (rec["skip"] == 0).astype(np.uint8)
        skipped += int(np.count_nonzero(rec["skip"]))
        rounds += 1
    assert dm.getNumClusters() == 0 and orc.n_clusters == 0
    np.testing.assert_array_equal(dm.downloadLabels(), orc.labels())
    ids, k = orc.final_partition()
    fp = dm.getFinalPartition()
    np.testing.assert_array_equal(fp.clusterIds, ids)
    np.testing.assert_array_equal(dm.downloadCertificates(), orc.certificates())
    _certified(g.offsets, g.cols, dm, fp)
    # the graph driver runs the same schedule
    gd = P.CudaDeviceManager()
    gd.set_schedule(_lib.SCHEDULE_LEARNED, model.weights, model.norm, **learn.SHIPPED_SCHEDULE)
    gd.initialize(g)
    gd.expanderDecomposition()
    np.testing.assert_array_equal(gd.getFinalPartition().clusterIds, ids)


def _stratified(params, count=32):
    order = sorted(range(len(params)), key=lambda i: (params[i][0], i))
    picks = {order[int(round(q * (len(order) - 1)))] for q in np.linspace(0.0, 1.0, count)}
    return sorted(picks)


def test_batch512_stratified_subset_bit_exact():
    params = B.sbm_batch_params(512, seed=1)
    subset = _stratified(params)
    assert len(subset) == 32 and max(params[i][0] for i in subset) == max(p[0] for p in params)
    off_d, cols_d, n, m, starts = B.sbm_batch(512, seed=1, instances=subset)
    off64 = off_d.to(__import__("torch").int64)
    off, cols = _host(off64, cols_d)
    dm = P.CudaDeviceManager()
    dm.initialize_batched_device(n, m, off64.data_ptr(), True, cols_d.data_ptr(), starts)
    x0 = dm.readRandomWalkValues()
    rounds = dm.expanderDecomposition()
    k0 = starts.shape[0] - 1
    labels = np.repeat(np.arange(k0, dtype=np.int32), np.diff(starts.astype(np.int64)))
    act = np.zeros(n, dtype=O.LNODE)
    act["nix"] = np.arange(n, dtype=np.uint32)
    act["label"] = labels
    orc = O.Oracle(off, cols, O.MODE_PXR, SC, RW)
    orc.set_state(labels, act, x0.astype(np.float64), np.diff(off.astype(np.int64)).astype(np.uint32), cols, k0, 0)
    _plain_against_oracle(off, cols, dm, rounds, orc)
