"""Expander hierarchy on the GPU: the consumer of the drop-in decomposition
(ExpanderHierarchy, lib/algorithms/expander_hierarchy.h:13-162).

The reference builds it on the host: decompose the current graph, contract
every cluster to a vertex (the cut edges become the next level's edges),
repeat until one vertex is left; its hook for an external decomposition,
``computeExpanderDecomposition<true>``, is empty (:91-101).  Here every level
is decomposed by this library and contracted on the device (pxr_contract);
the level graphs never leave device memory.

As in the reference, a level whose decomposition cuts more than 95 % of the
edges is decomposed again with the sweep threshold lowered by a factor 0.8
(:116-121).  The reference loops forever on a level with no edges and more
than one vertex (every vertex stays its own cluster); here such a level ends
the hierarchy with its vertices as roots.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .manager import CudaDeviceManager


@dataclass
class Level:
    n: int                  # vertices of the level graph
    m: int                  # edges of the level graph
    clusters: int           # clusters of its decomposition (vertices of the next level)
    cut_edges: int          # edges between them (edges of the next level)
    sc_threshold: float     # sweep threshold the decomposition used
    parents: np.ndarray     # per level-graph vertex, its cluster (vertex of the next level)
    volumes: np.ndarray     # per cluster, the volume of its subtree in the input graph
    cut_sizes: np.ndarray   # per cluster, the cut slots leaving it in the level graph


def _p(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


def contract(offsets, cols, ids, k: int, level_volumes=None, device: int = 0):
    """pxr_contract on device tensors: (offsets, cols, m, cut_sizes, volumes)."""
    import torch
    L = _lib.load()
    dev = torch.device("cuda", device)
    n = int(offsets.shape[0]) - 1
    slots = int(cols.shape[0])
    scratch = torch.empty(max(int(L.pxr_contract_scratch_bytes(slots)), 1), dtype=torch.uint8, device=dev)
    out_off = torch.empty(k + 1, dtype=torch.int32, device=dev)
    out_cols = torch.empty(max(slots, 1), dtype=torch.int32, device=dev)
    cut = torch.empty(k, dtype=torch.int64, device=dev)
    vol = torch.empty(k, dtype=torch.int64, device=dev)
    m = C.c_uint64(0)
    st = L.pxr_contract(n, _p(offsets), _p(cols) if slots else None, _p(ids), k,
                        _p(level_volumes) if level_volumes is not None else None, _p(scratch), _p(out_off),
                        _p(out_cols), C.byref(m), _p(cut), _p(vol),
                        C.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    if st != 0:
        raise _lib.PxrError(st, "pxr_contract")
    return out_off, out_cols[: 2 * m.value], m.value, cut, vol


def build(offsets, cols, seed: int = 6582, sc_threshold: float = 0.3, rw_threshold: float = 1e-4,
          device: int = 0, max_levels: int = 64) -> list[Level]:
    """The hierarchy of a graph given as device tensors (int32 offsets and
    columns): every level decomposed on the GPU, until one vertex is left."""
    import torch
    dev = torch.device("cuda", device)
    levels: list[Level] = []
    off, col = offsets.to(dev), cols.to(dev)
    vol_below = None
    sc = sc_threshold
    while int(off.shape[0]) - 1 > 1 and len(levels) < max_levels:
        n = int(off.shape[0]) - 1
        m = int(col.shape[0]) // 2
        dm = CudaDeviceManager(seed=seed, sc_threshold=sc, rw_threshold=rw_threshold, device=device)
        dm.initialize_device(n, m, off.data_ptr(), False, col.data_ptr())
        dm.expanderDecomposition()
        fp = dm.getFinalPartition()
        cut = dm.countCutEdges()
        dm.close()
        if m > 0 and cut > 0.95 * m:
            sc *= 0.8          # the reference's adjustment (expander_hierarchy.h:116-121)
            continue
        ids = torch.from_numpy(fp.clusterIds).to(dev)
        noff, ncol, nm, cut_sizes, vol = contract(off, col, ids, fp.numClusters, vol_below, device)
        levels.append(Level(n, m, fp.numClusters, nm, sc, fp.clusterIds, vol.cpu().numpy(), cut_sizes.cpu().numpy()))
        if fp.numClusters == n:
            break              # nothing merged (no edges left): the remaining vertices are roots
        off, col, vol_below = noff, ncol, vol
    return levels
