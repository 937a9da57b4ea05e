"""Graphs built on the GPU (pxr_rmat_edges, pxr_build_csr).

The CSR of an edge list is built with the library's own radix sort on the
device (self-loops dropped, duplicates merged, rows sorted), the GPU
counterpart of the reference's host-side DynamicGraph::finalize
(lib/core/graph.h:147-184).  ``rmat`` samples the same edges as
``graphs.rmat`` (same counter-based hash), so the two agree exactly; at
scale 24 the device build takes well under a second where numpy takes
minutes.  Device memory comes from torch (plumbing only).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .graphs import CSRGraph


def _p(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


def build_csr(n: int, u, v, device: int = 0):
    """(offsets, cols, m) as torch tensors on the device from edge tensors u, v (int32 views of uint32 ids)."""
    import torch
    L = _lib.load()
    dev = torch.device("cuda", device)
    n_edges = int(u.shape[0])
    scratch = torch.empty(max(int(L.pxr_build_csr_scratch_bytes(n_edges)), 1), dtype=torch.uint8, device=dev)
    offsets = torch.empty(n + 1, dtype=torch.int32, device=dev)
    cols = torch.empty(max(2 * n_edges, 1), dtype=torch.int32, device=dev)
    m = C.c_uint64(0)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    st = L.pxr_build_csr(n, n_edges, _p(u) if n_edges else None, _p(v) if n_edges else None, _p(scratch),
                         _p(offsets), _p(cols), C.byref(m), stream)
    if st != 0:
        raise _lib.PxrError(st, "pxr_build_csr")
    return offsets, cols[: 2 * m.value], m.value


def build_csr_finalize(n: int, u, v, device: int = 0):
    """(offsets, cols, m) on the device with the reference's finalize
    semantics (pxr_build_csr_finalize): duplicates and self-loops kept, both
    directions, rows sorted; m = number of input edges."""
    import torch
    L = _lib.load()
    dev = torch.device("cuda", device)
    n_edges = int(u.shape[0])
    scratch = torch.empty(max(int(L.pxr_build_csr_scratch_bytes(n_edges)), 1), dtype=torch.uint8, device=dev)
    offsets = torch.empty(n + 1, dtype=torch.int32, device=dev)
    cols = torch.empty(max(2 * n_edges, 1), dtype=torch.int32, device=dev)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    st = L.pxr_build_csr_finalize(n, n_edges, _p(u) if n_edges else None, _p(v) if n_edges else None, _p(scratch),
                                  _p(offsets), _p(cols), stream)
    if st != 0:
        raise _lib.PxrError(st, "pxr_build_csr_finalize")
    return offsets, cols[: 2 * n_edges], n_edges


def mtx_header(data: bytes):
    """(rows, n, n_edges, body offset) of a Matrix Market file's bytes: comment
    lines start with '%'; the first other line holds three integers, of which
    readDynGraph (lib/utils/graph_io.h:49-84) takes the second as the vertex
    count and the third as the edge count."""
    pos = 0
    while True:
        end = data.find(b"\n", pos)
        line = data[pos:] if end < 0 else data[pos:end]
        if not line.lstrip().startswith(b"%"):
            fields = line.split()
            if len(fields) < 3:
                raise ValueError("Matrix Market size line needs three integers")
            return int(fields[0]), int(fields[1]), int(fields[2]), (len(data) if end < 0 else end + 1)
        if end < 0:
            raise ValueError("no size line")
        pos = end + 1


def read_mtx(path, device: int = 0):
    """A Matrix Market graph read as the reference's readDynGraph +
    DynamicGraph::finalize read it, with the body tokenised and the CSR built
    on the device: (offsets, cols, n, m) as torch tensors / ints."""
    import torch
    L = _lib.load()
    dev = torch.device("cuda", device)
    with open(path, "rb") as f:
        data = f.read()
    _, n, n_edges, body = mtx_header(data)
    text = torch.frombuffer(bytearray(data[body:]) if body < len(data) else bytearray(1), dtype=torch.uint8)
    text_d = text.to(dev)
    nbytes = len(data) - body
    u = torch.empty(max(n_edges, 1), dtype=torch.int32, device=dev)
    v = torch.empty(max(n_edges, 1), dtype=torch.int32, device=dev)
    scratch = torch.empty(max(int(L.pxr_parse_mtx_scratch_bytes(nbytes)), 1), dtype=torch.uint8, device=dev)
    tokens = C.c_uint64(0)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    st = L.pxr_parse_mtx_body(_p(text_d), nbytes, n, n_edges, _p(u), _p(v), _p(scratch), C.byref(tokens), stream)
    if st != 0:
        raise _lib.PxrError(st, f"pxr_parse_mtx_body ({tokens.value} numbers for {n_edges} edges)")
    del text_d, scratch
    offsets, cols, m = build_csr_finalize(n, u[:n_edges], v[:n_edges], device)
    return offsets, cols, n, m


def rmat_edges(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19, seed: int = 1,
               device: int = 0):
    import torch
    L = _lib.load()
    dev = torch.device("cuda", device)
    samples = edge_factor << scale
    u = torch.empty(samples, dtype=torch.int32, device=dev)
    v = torch.empty(samples, dtype=torch.int32, device=dev)
    st = L.pxr_rmat_edges(scale, samples, a, b, c, seed, _p(u), _p(v),
                          C.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    if st != 0:
        raise _lib.PxrError(st, "pxr_rmat_edges")
    return u, v


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19, seed: int = 1,
         device: int = 0):
    """R-MAT CSR on the device: (offsets, cols, n, m)."""
    u, v = rmat_edges(scale, edge_factor, a, b, c, seed, device)
    n = 1 << scale
    offsets, cols, m = build_csr(n, u, v, device)
    del u, v
    return offsets, cols, n, m


def to_host(offsets, cols, name: str = "") -> CSRGraph:
    return CSRGraph(offsets.cpu().numpy().view(np.uint32).copy(), cols.cpu().numpy().view(np.uint32).copy(), name)


def sbm_batch_params(count: int = 512, seed: int = 1, n_lo: float = 1e3, n_hi: float = 1e6, scale: float = 1.0):
    """Per-instance (n, blocks, d_in, d_out), drawn as graphs.sbm_batch draws them."""
    import math
    out = []
    for i in range(count):
        rng = np.random.default_rng([seed, i])
        n = max(4, int(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi))) * scale))
        blocks = int(rng.integers(2, 65))
        blocks = min(blocks, max(1, n // 2))
        d_in = float(rng.uniform(4, 32))
        d_out = float(rng.uniform(0.1, 2))
        out.append((n, blocks, d_in, d_out))
    return out


def sbm_batch_tasks(params, segment_len: int = 1 << 24, instances=None):
    """The work list of the device planted-partition sampler for instances
    `params` ((n, blocks, d_in, d_out) each, as sbm_batch_params), or for the
    subset `instances` of them (a shard): one task per block pair
    (SBM_TASK_DTYPE: vertex bases, block sizes, Bernoulli p, intra flag, and
    the key of the task in the whole batch, so a shard draws the same edges),
    the first global segment of every task (n_tasks + 1 entries, segments of
    segment_len candidate pairs), and the instance starts."""
    first_key = np.concatenate([[0], np.cumsum([b * (b + 1) // 2 for _, b, _, _ in params])])
    chosen = range(len(params)) if instances is None else instances
    tasks = []
    starts = [0]
    for i in chosen:
        n, blocks, d_in, d_out = params[i]
        key = int(first_key[i])
        base = starts[-1]
        bsz = n // blocks
        sizes = [bsz] * blocks
        sizes[-1] += n - bsz * blocks
        bstart = np.concatenate([[0], np.cumsum(sizes)]) + base
        p_in = d_in / max(bsz - 1, 1)
        p_out = d_out / max(n - bsz, 1)
        for a in range(blocks):
            tasks.append((bstart[a], bstart[a], sizes[a], sizes[a], min(p_in, 1.0), 1, key))
            key += 1
            for b in range(a + 1, blocks):
                tasks.append((bstart[a], bstart[b], sizes[a], sizes[b], min(p_out, 1.0), 0, key))
                key += 1
        starts.append(base + n)
    T = np.zeros(len(tasks), dtype=_lib.SBM_TASK_DTYPE)
    arr = np.asarray(tasks, dtype=np.float64)
    T["base_u"], T["base_v"] = arr[:, 0], arr[:, 1]
    T["su"], T["sv"], T["p"], T["intra"], T["key"] = arr[:, 2], arr[:, 3], arr[:, 4], arr[:, 5], arr[:, 6]
    su, sv = T["su"].astype(np.uint64), T["sv"].astype(np.uint64)
    cand = np.where(T["intra"] == 1, su * (su - np.uint64(1)) // np.uint64(2), su * sv)
    nseg = (cand + np.uint64(segment_len - 1)) // np.uint64(segment_len)
    prefix = np.zeros(len(tasks) + 1, dtype=np.uint64)
    np.cumsum(nseg, out=prefix[1:])
    return T, prefix, starts


def shard_instances(params, world: int):
    """Instances of a batch split over `world` ranks: longest expected edge
    count first, each to the rank with the fewest expected edges so far
    (ties to the lower rank); every rank's list in increasing instance order."""
    load = [0.0] * world
    shards = [[] for _ in range(world)]
    weight = [n * (d_in + d_out) / 2.0 for n, _, d_in, d_out in params]
    for i in sorted(range(len(params)), key=lambda i: (-weight[i], i)):
        r = min(range(world), key=lambda q: (load[q], q))
        shards[r].append(i)
        load[r] += weight[i]
    return [sorted(s) for s in shards]


def sbm_batch(count: int = 512, seed: int = 1, n_lo: float = 1e3, n_hi: float = 1e6, scale: float = 1.0,
              device: int = 0, segment_len: int = 1 << 24, instances=None):
    """Disjoint union of planted-partition instances built on the device:
    (offsets, cols, n, m, instance_start).  Instance parameters as
    graphs.sbm_batch; edges drawn on the device (pxr_sbm_edges), so the edge
    sample differs from the host generator's while following the same
    distribution (Bernoulli pairs, p_in = d_in / (b - 1), p_out = d_out / (n - b)).
    `instances`: build only these instances of the batch (a shard; each draws
    the same edges as in the whole batch)."""
    import torch
    L = _lib.load()
    dev = torch.device("cuda", device)
    params = sbm_batch_params(count, seed, n_lo, n_hi, scale)
    T, prefix, starts = sbm_batch_tasks(params, segment_len, instances)
    n_segments = int(prefix[-1])
    d_tasks = torch.from_numpy(T.view(np.uint8).copy()).to(dev)
    d_prefix = torch.from_numpy(prefix.view(np.int64).copy()).to(dev)
    d_count = torch.zeros(max(n_segments, 1), dtype=torch.int32, device=dev)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    st = L.pxr_sbm_edges(_p(d_tasks), len(T), _p(d_prefix), n_segments, segment_len, seed, _p(d_count), None,
                         None, None, stream)
    if st != 0:
        raise _lib.PxrError(st, "pxr_sbm_edges (count)")
    counts = d_count[:n_segments].to(torch.int64)
    offs = torch.zeros(max(n_segments, 1), dtype=torch.int64, device=dev)
    if n_segments > 1:
        offs[1:n_segments] = torch.cumsum(counts, 0)[:-1]
    total = int(counts.sum().item()) if n_segments else 0
    u = torch.empty(max(total, 1), dtype=torch.int32, device=dev)
    v = torch.empty(max(total, 1), dtype=torch.int32, device=dev)
    st = L.pxr_sbm_edges(_p(d_tasks), len(T), _p(d_prefix), n_segments, segment_len, seed, None, _p(offs),
                         _p(u), _p(v), stream)
    if st != 0:
        raise _lib.PxrError(st, "pxr_sbm_edges (write)")
    del d_count, offs
    n_total = starts[-1]
    offsets, cols, m = build_csr(n_total, u[:total], v[:total], device)
    return offsets, cols, n_total, m, np.asarray(starts, dtype=np.uint32)
