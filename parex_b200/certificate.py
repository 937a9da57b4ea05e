"""End-to-end certificate check of a decomposition's output.

A cluster leaves the decomposition only through the reference's keep test
(KeepClusterFlagOp, cuda/devPartition.h:173-184): it is certified when its
potential spread max(x) - min(x) is below rw_threshold or it has fewer than
two vertices.  When the certified set is exactly the set the round swept, the
exact sweep of that round also found no prefix with sparsity below
sc_threshold (CheckThreshold, cuda/devSweepCut.h:321-331); otherwise it is a
piece of a cluster that was cut (or split into components) in that round.

This module checks both from the output alone, independently of the code that
made the decisions:

* the potentials of a certified vertex are frozen from the round of its
  certificate on (inactive vertices neither walk nor recentre), so the final
  potentials are the ones the keep test saw;
* the certificate record (``CudaDeviceManager.downloadCertificates``) gives per
  vertex the round of its certificate and whether its set was swept whole;
  certified clusters are the vertex sets sharing (final id, round) - final ids
  alone can merge clusters of different rounds that reused a negative label,
  as the reference's getFinalPartition does;
* the sweep of a certified cluster is recomputed from scratch on the original
  graph: vertices ordered by (potential, vertex id), prefix cut edges and
  prefix volumes over the cluster's induced edges, sparsity
  cut / min(vol, total - vol) in float (2 where the denominator is 0), and its
  minimum compared with sc_threshold;
* the reference's cluster invariants (tests/clusterTest.cpp:11-40) restated on
  the output: every certified cluster is connected through its own edges, and
  (given the library's internal degrees) a whole-swept cluster's internal
  degrees are its induced degrees;
* cut edges are recounted from the final ids (edges whose ends carry
  different ids), the count the reference's application makes on the host
  with Partition::splitByIndices (main.cpp:54-60).

The arithmetic is torch tensor code, so it runs on the CPU for small graphs
and on the GPU for the benchmark's graphs.
"""
from __future__ import annotations

import numpy as np

CUT_BIT = 0x80000000


def _tensor(a, device, dtype=None):
    import torch
    if isinstance(a, torch.Tensor):
        t = a.to(device)
    else:
        arr = np.ascontiguousarray(a)
        if arr.dtype == np.uint32:
            arr = arr.astype(np.int64)
        elif arr.dtype == np.uint64:
            arr = arr.view(np.int64)
        t = torch.from_numpy(arr).to(device)
    return t.to(dtype) if dtype is not None else t


def _ordered_bits(x):
    """Monotone map of float32 values onto int64 keys (the sort key's potential part)."""
    import torch
    b = x.contiguous().view(torch.int32).to(torch.int64) & 0xFFFFFFFF
    neg = b >= 0x80000000
    return torch.where(neg, b ^ 0xFFFFFFFF, b ^ 0x80000000)


def check(offsets, cols, final_ids, x, cert, sc_threshold: float = 0.3, rw_threshold: float = 1e-4,
          device=None, connectivity: bool = True, degrees=None, max_label_rounds: int = 100000) -> dict:
    """Check every certified cluster of a finished decomposition.

    offsets, cols: the ORIGINAL graph (before edge disabling), CSR.
    final_ids: FinalPartition ids (int32[n]); x: final potentials (float32[n]);
    cert: certificate record (uint32[n]); degrees: the library's internal
    degrees after the decomposition (downloadDegrees), optional.
    Returns counts; ``ok`` is True when every vertex is certified, every
    certified cluster passes the walk-threshold test, every whole-swept one has
    no sweep prefix below sc_threshold, and (with ``connectivity``) every one
    is connected.
    """
    import torch
    dev = torch.device(device) if device is not None else torch.device("cpu")
    off = _tensor(offsets, dev, torch.int64)
    n = int(off.shape[0]) - 1
    col = _tensor(cols, dev, torch.int64)
    fid = _tensor(final_ids, dev, torch.int64)
    xs = _tensor(np.ascontiguousarray(x, dtype=np.float32) if not isinstance(x, torch.Tensor) else x, dev,
                 torch.float32)
    ce = _tensor(cert, dev, torch.int64) & 0xFFFFFFFF
    rep = {"vertices": n, "uncertified_vertices": int((ce == 0).sum().item())}
    if n == 0:
        rep.update(clusters=0, threshold_violations=0, sweep_checked=0, sweep_violations=0,
                   min_sweep_sparsity=None, disconnected=0, degree_mismatches=0, cut_edges=0,
                   potential_ties=0, ok=rep["uncertified_vertices"] == 0)
        return rep

    tag = ce & 0x7FFFFFFF
    whole = (ce & CUT_BIT) == 0
    # certified clusters: (final id, certificate round)
    key = fid * (int(tag.max().item()) + 1) + tag
    _, gid = torch.unique(key, return_inverse=True)
    k = int(gid.max().item()) + 1
    size = torch.bincount(gid, minlength=k)

    # walk-threshold test on the frozen potentials (float max - min, as the keep test)
    xmax = torch.full((k,), -float("inf"), device=dev).scatter_reduce(0, gid, xs, "amax", include_self=True)
    xmin = torch.full((k,), float("inf"), device=dev).scatter_reduce(0, gid, xs, "amin", include_self=True)
    spread = xmax - xmin
    rw = torch.tensor(rw_threshold, dtype=torch.float32, device=dev)
    ok_walk = (spread < rw) | (size < 2)
    certified = torch.zeros(k, dtype=torch.bool, device=dev).scatter_(0, gid[tag > 0], True)
    rep["clusters"] = k
    rep["threshold_violations"] = int((certified & ~ok_walk).sum().item())

    # induced edges of every certified cluster
    deg = off[1:] - off[:-1]
    src = torch.repeat_interleave(torch.arange(n, device=dev), deg)
    rep["cut_edges"] = int((fid[src] != fid[col]).sum().item()) // 2
    inside = gid[src] == gid[col]
    s_in, d_in = src[inside], col[inside]
    del src, inside
    ideg = torch.bincount(s_in, minlength=n)
    vol = torch.zeros(k, dtype=torch.int64, device=dev).index_add_(0, gid, ideg)
    # clusterTest's internalDegree == |valid range|: a whole-swept certified
    # cluster's rows were last rescanned when it was formed, so the library's
    # internal degrees are its induced degrees
    rep["degree_mismatches"] = 0
    if degrees is not None:
        dg = _tensor(degrees, dev, torch.int64)
        rep["degree_mismatches"] = int(((dg != ideg) & whole & (tag > 0)).sum().item())

    # the exact sweep of every whole-swept certified cluster: order by
    # (cluster, potential, vertex id); prefix cut = sum of (later - earlier)
    # neighbours; prefix volume = sum of internal degrees
    ob = _ordered_bits(xs)
    order = torch.argsort(ob, stable=True)
    order = order[torch.argsort(gid[order], stable=True)]
    pos = torch.empty(n, dtype=torch.int64, device=dev)
    pos[order] = torch.arange(n, device=dev)
    diff = torch.zeros(n, dtype=torch.int64, device=dev).index_add_(
        0, s_in, torch.where(pos[d_in] > pos[s_in], 1, -1).to(torch.int64))
    g_sorted = gid[order]
    cdif = torch.cumsum(diff[order], 0)
    cvol = torch.cumsum(ideg[order], 0)
    start = torch.zeros(k, dtype=torch.int64, device=dev)
    start[1:] = torch.cumsum(size, 0)[:-1]
    base_dif = torch.where(start > 0, cdif[(start - 1).clamp(min=0)], torch.zeros_like(start))
    base_vol = torch.where(start > 0, cvol[(start - 1).clamp(min=0)], torch.zeros_like(start))
    pdif = cdif - base_dif[g_sorted]
    pvol = cvol - base_vol[g_sorted]
    tot = vol[g_sorted]
    denom = torch.where(pvol >= tot, torch.zeros_like(pvol), torch.minimum(pvol, tot - pvol))
    num = (pdif & 0xFFFFFFFF).to(torch.float32)   # the sweep divides the 32-bit pattern
    sp = torch.where(denom > 0, num / denom.to(torch.float32).clamp(min=1.0), torch.full_like(num, 2.0))
    best = torch.full((k,), 2.0, device=dev).scatter_reduce(0, g_sorted, sp, "amin", include_self=True)
    swept_whole = torch.zeros(k, dtype=torch.bool, device=dev).scatter_(0, gid[whole & (tag > 0)], True)
    sc = torch.tensor(sc_threshold, dtype=torch.float32, device=dev)
    rep["sweep_checked"] = int(swept_whole.sum().item())
    rep["sweep_violations"] = int((swept_whole & (best < sc)).sum().item())
    rep["min_sweep_sparsity"] = float(best[swept_whole].min().item()) if rep["sweep_checked"] else None
    # exact potential ties inside a cluster: there the reference's sort keeps
    # its previous order rather than vertex order, so a prefix may differ
    same = (g_sorted[1:] == g_sorted[:-1]) & (ob[order][1:] == ob[order][:-1])
    rep["potential_ties"] = int(same.sum().item())
    del pos, diff, cdif, cvol, pdif, pvol, tot, denom, num, sp, order

    # connectivity: min-label propagation over induced edges with pointer jumping
    rep["disconnected"] = 0
    if connectivity:
        lab = torch.arange(n, device=dev)
        for _ in range(max_label_rounds):
            nb_min = lab.clone().scatter_reduce_(0, s_in, lab[d_in], "amin", include_self=True)
            nxt = torch.minimum(lab, nb_min)
            nxt = nxt[nxt]
            if torch.equal(nxt, lab):
                break
            lab = nxt
        roots = torch.bincount(gid[lab == torch.arange(n, device=dev)], minlength=k)
        rep["disconnected"] = int((roots > 1).sum().item())
    rep["ok"] = (rep["uncertified_vertices"] == 0 and rep["threshold_violations"] == 0
                 and rep["sweep_violations"] == 0 and rep["disconnected"] == 0
                 and rep["degree_mismatches"] == 0)
    return rep
