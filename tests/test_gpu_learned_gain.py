"""What the shipped stop predictor (parex_b200/data/stop_predictor.npz) gains
over the plain method, on held-out graphs (seeds the training traces never
saw):

* fewer swept vertices than the plain method (the work the schedule skips);
* cut edges (edges between output clusters, the recount main.cpp:54-60
  makes) within 2 % of the plain method's;
* every output cluster certified (parex_b200/certificate.py): the network
  never certifies or cuts on its own;
* the audit mode's false-stop rate (skipped sweeps that would have cut) is
  reported, and the audit gives the learned partition unchanged.
"""
import numpy as np
import pytest

import parex_b200 as P
from parex_b200 import _lib, certificate as CERT, graphs as G, learn

pytestmark = pytest.mark.gpu

SC, RW = 0.3, 1e-4

# graphs and seeds that no training trace used; the planted partition and the
# grid are cut in many places, R-MAT graphs hardly at all (their giant
# component certifies by mixing)
HELD_OUT = {
    "rmat18_seed101": lambda: G.rmat(18, 16, seed=101),
    "sbm16k_seed6583": lambda: G.sbm_graph(16384, 16, 12.0, 0.5, 6583),
    "sbm32k_seed77": lambda: G.sbm_graph(32768, 32, 12.0, 0.5, 77),
}


def _run(g, mode, model):
    dm = P.CudaDeviceManager()
    if mode != _lib.SCHEDULE_PLAIN:
        dm.set_schedule(mode, model.weights, model.norm, **learn.SHIPPED_SCHEDULE)
    dm.initialize(g)
    rounds = dm.expanderDecomposition()
    fp = dm.getFinalPartition()
    st = dm.stats()
    rep = CERT.check(g.offsets, g.cols, fp.clusterIds, dm.readRandomWalkValues(), dm.downloadCertificates(),
                     SC, RW, device="cuda")
    return {"rounds": rounds, "ids": fp.clusterIds, "cut": dm.countCutEdges(), "swept": st["swept_items"],
            "skipped": st["skipped_sweeps"], "false_stops": st["false_stops"], "cert": rep}


@pytest.mark.parametrize("name", sorted(HELD_OUT))
def test_trained_network_gains_over_plain(name, record_property):
    g = HELD_OUT[name]()
    model = learn.Model.load()
    plain = _run(g, _lib.SCHEDULE_PLAIN, None)
    learned = _run(g, _lib.SCHEDULE_LEARNED, model)
    audit = _run(g, _lib.SCHEDULE_AUDIT, model)
    assert plain["cert"]["ok"], plain["cert"]
    assert learned["cert"]["ok"], learned["cert"]
    assert learned["swept"] < plain["swept"]
    assert abs(learned["cut"] - plain["cut"]) <= 0.02 * max(plain["cut"], 1)
    np.testing.assert_array_equal(audit["ids"], learned["ids"])
    rate = audit["false_stops"] / max(audit["skipped"], 1)
    record_property("swept_ratio", learned["swept"] / plain["swept"])
    record_property("false_stop_rate", rate)
    record_property("cut_plain", plain["cut"])
    record_property("cut_learned", learned["cut"])
    print(f"{name}: swept {learned['swept']}/{plain['swept']} = {learned['swept'] / plain['swept']:.3f}, "
          f"cut {learned['cut']}/{plain['cut']}, rounds {learned['rounds']}/{plain['rounds']}, "
          f"false-stop rate {rate:.4f} ({audit['false_stops']} of {audit['skipped']} skipped sweeps)")
