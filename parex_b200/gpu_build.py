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
