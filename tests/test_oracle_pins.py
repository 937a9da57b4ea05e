"""Pins of the CPU oracle against fixtures recorded from the reference's own GPU
binary (tests/golden/make_golden.py).  The oracle runs in ORC_MODE_REF
(double potentials, as the reference) and is fed the reference's recorded
state before every stage, so each stage is compared on identical inputs.

Bars:
* walk: |x_oracle - x_ref| <= 1e-12 * max |x_ref| over the active vertices;
* sort order and prefix sums (NodeData): bit-exact;
* per-cluster argmin: bit-exact, except where the reference's fast-math
  division breaks an exact tie of ratios (the oracle divides exactly); each
  such case must be a tie under exact division;
* labels after cut / components / relabel, internal degrees, disabled slots:
  bit-exact;
* recentred potentials: within 1e-6 * max |x| (the reference's per-cluster sum
  is a float reduction in Thrust's order);
* x0: within 4 float ulps (the oracle's inverse erfc is its own).
"""
import numpy as np
import pytest

from conftest import unpack_valid
from oracle import oracle as O

TRACED = ["sbm2k", "grid16"]


def _state(fx, r):
    cols = unpack_valid(fx[f"r{r}_valid_pre"], fx["cols"])
    return fx[f"r{r}_lab_pre"], fx[f"r{r}_act_pre"], fx[f"r{r}_x_pre"], fx[f"r{r}_deg_pre"], cols


def _exact_ratio(edge_diff, denom):
    return np.float32(np.uint32(edge_diff)) / np.float32(denom) if denom else np.float32(2.0)


@pytest.mark.parametrize("name", TRACED)
def test_initial_potentials_within_4_ulps(golden, name):
    fx = golden["trace"](name)
    x0 = O.initial_potentials(fx["offsets"], 6582)
    ref = fx["x0"]
    ulp = np.spacing(np.abs(ref))
    assert np.all(np.abs(x0.astype(np.float64) - ref) <= 4 * ulp)
    assert np.mean(x0 == ref) > 0.5


@pytest.mark.parametrize("name", TRACED)
def test_oracle_stages_match_reference_trace(golden, name):
    fx = golden["trace"](name)
    meta = golden["summary"]["graphs"][name]["meta"]
    rounds = golden["summary"]["graphs"][name]["rounds_kept"]
    orc = O.Oracle(fx["offsets"], fx["cols"], O.MODE_REF)
    approx_ties = 0
    for r in rounds:
        mt = meta[str(r)]
        lab, act, x, deg, cols = _state(fx, r)
        prev_keep = meta[str(r - 1)]["k_keep"] if r > 1 else 1
        orc.set_state(lab, act, x, deg, cols, prev_keep, 0)
        # walk step from the reference's potentials
        orc.walk()
        xw = fx[f"r{r}_x_walk"]
        sel = act["nix"][act["label"] >= 0]
        xo = orc.potentials()
        assert np.max(np.abs(xo[sel] - xw[sel])) <= 1e-12 * np.max(np.abs(xw[sel]))
        # sweep from the reference's post-walk potentials
        orc.set_potentials(xw)
        orc.rekey()
        orc.sweep()
        assert orc.n_active == mt["n_post"]
        assert orc.smallest_label == mt["smallest"]
        np.testing.assert_array_equal(orc.sorted(), fx[f"r{r}_sorted"])
        oc, rc = orc.all_cuts(), fx[f"r{r}_allcuts"]
        np.testing.assert_array_equal(oc["label"], rc["label"])
        srt, vols = orc.sorted(), orc.sweep_volumes()
        act_s = orc.active()
        for c in np.nonzero((oc["offset"] != rc["offset"]) | (oc["sparsity"] != rc["sparsity"]))[0]:
            # the reference's pick must be an exact-division tie with the oracle's
            idx = np.nonzero(act_s["label"] == oc["label"][c])[0]
            j = idx[rc["offset"][c] - 1]
            tot = vols[c]
            pv = srt["prefix_volume"][j]
            den = 0 if pv >= tot else min(pv, tot - pv)
            assert _exact_ratio(srt["prefix_edge_diff"][j], den) == oc["sparsity"][c]
            assert abs(float(rc["sparsity"][c]) - float(oc["sparsity"][c])) <= 2 * np.spacing(oc["sparsity"][c])
            approx_ties += 1
        if mt["n_post"] == 0:
            continue
        # downstream stages from the reference's cuts
        cut_same = np.array_equal(oc[oc["sparsity"] < 0.3]["offset"], rc[rc["sparsity"] < 0.3]["offset"])
        if not cut_same:
            continue
        orc.cut_stage()
        np.testing.assert_array_equal(orc.labels(), fx[f"r{r}_lab_cut"])
        orc.components_stage()
        np.testing.assert_array_equal(orc.labels(), fx[f"r{r}_lab_cc"])
        orc.cluster_data_stage()
        np.testing.assert_array_equal(orc.data_labels(), fx[f"r{r}_clabels"])
        cd, rcd = orc.cluster_values(), fx[f"r{r}_cdata"]
        for f in ("max", "min", "count"):
            np.testing.assert_array_equal(cd[f], rcd[f])
        orc.recenter_stage()
        np.testing.assert_array_equal(orc.labels(), fx[f"r{r}_lab_final"])
        xf = fx[f"r{r}_x_final"]
        keep = orc.active()
        ks = keep["nix"][keep["label"] >= 0]
        if ks.size:
            assert np.max(np.abs(orc.potentials()[ks] - xf[ks])) <= 1e-6 * np.max(np.abs(xf[ks]))
        orc.disable_stage()
        np.testing.assert_array_equal(orc.internal_degrees(), fx[f"r{r}_deg_final"])
        np.testing.assert_array_equal(orc.cols(), unpack_valid(fx[f"r{r}_valid_final"], fx["cols"]))
    # the fast-math near-ties are rare
    assert approx_ties <= 60


@pytest.mark.parametrize("name", TRACED)
def test_negative_label_reuse_matches_reference(golden, name):
    """The reference restarts negative labels at -1 after a round without
    deactivations (d_smallestLabel is the smallest label in the sort,
    cuda/devSweepCut.h:530-537), so certified clusters of different rounds can
    share a label; the oracle does the same."""
    meta = golden["summary"]["graphs"][name]["meta"]
    smallest = [meta[str(r)]["smallest"] for r in range(1, len(meta) + 1) if str(r) in meta]
    assert 0 in smallest[1:]
    orc = O.Oracle(*_graph(golden, name), O.MODE_REF)
    fx = golden["trace"](name)
    orc.set_potentials(fx["x0"].astype(np.float64))
    orc.decompose()
    ids, k = orc.final_partition()
    assert k == len(np.unique(orc.labels()))


def _graph(golden, name):
    fx = golden["trace"](name)
    return fx["offsets"], fx["cols"]


@pytest.mark.parametrize("name", TRACED)
def test_reference_mode_end_to_end_band(golden, name):
    """Whole decomposition in ORC_MODE_REF from the reference's x0: cluster count
    and cut edges within 5 % of the reference binary's."""
    fx = golden["trace"](name)
    orc = O.Oracle(fx["offsets"], fx["cols"], O.MODE_REF)
    orc.set_potentials(fx["x0"].astype(np.float64))
    orc.decompose()
    ids, k = orc.final_partition()
    ref = golden["summary"]["graphs"][name]["reference_gpu"]
    assert abs(k - ref["num_clusters_fp"]) <= 0.05 * ref["num_clusters_fp"]
    assert abs(orc.num_cut_edges() - ref["cut_edges_device"]) <= 0.05 * ref["cut_edges_device"]
