"""Python mirror of the reference's drop-in class CudaDeviceManager (cuda/interface.h:16-57).

Method names, argument meaning and return values follow the reference:

=========================  =====================================================
reference member            here
=========================  =====================================================
initialize(const Graph&)    initialize(graph)  (a CSRGraph or (offsets, cols))
downloadGraph()             downloadGraph() -> (offsets, cols), disabled = 0xFFFFFFFF
downloadDegrees()           downloadDegrees() -> internal degrees (uint32[n])
downloadPartition()         downloadPartition() -> NodeData records in sweep order
iterateRandomWalk()         iterateRandomWalk()
readRandomWalkValues()      readRandomWalkValues() -> float32[n]
computeSweepCuts()          computeSweepCuts()
readSweepCuts()             readSweepCuts() -> AllSweepCuts(clusterIds, cuts)
cutClusters()               cutClusters()
getNumCutEdges()            getNumCutEdges()
expanderDecomposition()     expanderDecomposition() -> rounds run
getFinalPartition()         getFinalPartition() -> FinalPartition(clusterIds, numClusters)
downloadActiveEdgeMap()     downloadActiveEdgeMap() -> int32[2m]
downloadLabels()            downloadLabels() -> int32[n]
getNumClusters()            getNumClusters() (the reference returns 0; here the
                            number of active clusters)
updateLabels(...)           updateLabels(...) (a no-op, as in cuda/devGraph.h:191-206)
=========================  =====================================================

Two members have no counterpart in the class: ``countCutEdges()`` recounts
the cut edges of the final partition on the device (the count main.cpp:54-60
makes on the host after getFinalPartition), and ``downloadCertificates()``
returns the certificate record that parex_b200/certificate.py checks.

Errors raise ``PxrError`` carrying the C status; the reference has no error
reporting at all.
"""
from __future__ import annotations

import ctypes as C
from typing import NamedTuple

import numpy as np

from . import _lib
from .graphs import CSRGraph

NODE_DATA = np.dtype([("nix", "<u4"), ("prefix_volume", "<u4"), ("prefix_edge_diff", "<i4"),
                      ("offset_in_cluster", "<u4")])
SWEEP_CUT = np.dtype([("label", "<i4"), ("sparsity", "<f4"), ("offset", "<u4")])


class AllSweepCuts(NamedTuple):
    clusterIds: np.ndarray
    cuts: np.ndarray


class FinalPartition(NamedTuple):
    clusterIds: np.ndarray
    numClusters: int


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class CudaDeviceManager:
    """One decomposition on one GPU; not thread-safe (like the reference)."""

    def __init__(self, seed: int = 6582, sc_threshold: float = 0.3, rw_threshold: float = 1e-4,
                 max_rounds: int = 200000, device: int = 0, division: int = _lib.DIV_IEEE,
                 driver: int = _lib.DRIVER_GRAPH, tune: int = _lib.TUNE_AUTO,
                 components: int = _lib.COMPONENTS_AUTO, memory_cap_mib: int = 0):
        L = _lib.load()
        cfg = _lib.Config()
        L.pxr_config_default(C.byref(cfg))
        cfg.seed = seed
        cfg.sc_threshold = sc_threshold
        cfg.rw_threshold = rw_threshold
        cfg.max_rounds = max_rounds
        cfg.device = device
        cfg.division = division
        cfg.driver = driver
        cfg.tune = tune
        cfg.components = components
        cfg.memory_cap_mib = memory_cap_mib
        self._h = C.c_void_p()
        _lib.check(None, L.pxr_create(C.byref(cfg), C.byref(self._h)))
        self._L = L
        self.n = 0
        self.m = 0

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._L.pxr_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _call(self, fn, *args):
        _lib.check(self._h, fn(self._h, *args))

    # -- reference members ------------------------------------------------
    def initialize(self, graph) -> None:
        if isinstance(graph, CSRGraph):
            offsets, cols = graph.offsets, graph.cols
        else:
            offsets, cols = graph
        cols = np.ascontiguousarray(cols, dtype=np.uint32)
        n = int(offsets.shape[0] - 1)
        m = int(cols.shape[0] // 2)
        if offsets.dtype == np.uint64 or 2 * m >= 2**32:
            off = np.ascontiguousarray(offsets, dtype=np.uint64)
            self._call(self._L.pxr_initialize64, n, m, _ptr(off), _ptr(cols))
        else:
            off = np.ascontiguousarray(offsets, dtype=np.uint32)
            self._call(self._L.pxr_initialize, n, m, _ptr(off), _ptr(cols))
        self.n, self.m = n, m

    def initialize_batched(self, graph, instance_start) -> None:
        """Disjoint union of independent instances, each its own starting
        cluster (pxr_initialize_batched); ``instance_start`` has one entry per
        instance plus the final n."""
        if isinstance(graph, CSRGraph):
            offsets, cols = graph.offsets, graph.cols
        else:
            offsets, cols = graph
        cols = np.ascontiguousarray(cols, dtype=np.uint32)
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        starts = np.ascontiguousarray(instance_start, dtype=np.uint32)
        n = int(off.shape[0] - 1)
        m = int(cols.shape[0] // 2)
        self._call(self._L.pxr_initialize_batched, n, m, _ptr(off), _ptr(cols), int(starts.shape[0] - 1),
                   _ptr(starts))
        self.n, self.m = n, m

    def initialize_batched_device(self, n: int, m: int, offsets_ptr: int, offsets_are_64bit: bool, cols_ptr: int,
                                  instance_start) -> None:
        """initialize_batched() from a CSR already in device memory."""
        starts = np.ascontiguousarray(instance_start, dtype=np.uint32)
        self._call(self._L.pxr_initialize_batched_device, n, m, C.c_void_p(offsets_ptr), 1 if offsets_are_64bit else 0,
                   C.c_void_p(cols_ptr), int(starts.shape[0] - 1), _ptr(starts))
        self.n, self.m = n, m

    def iterateRandomWalk(self) -> None:
        self._call(self._L.pxr_walk_step)

    def computeSweepCuts(self) -> None:
        self._call(self._L.pxr_sweep)

    def cutClusters(self) -> None:
        self._call(self._L.pxr_cut_clusters)

    def expanderDecomposition(self) -> int:
        rounds = C.c_uint32(0)
        self._call(self._L.pxr_decompose, C.byref(rounds))
        return int(rounds.value)

    def readRandomWalkValues(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=np.float32)
        self._call(self._L.pxr_read_potentials, _ptr(out))
        return out

    def readSweepCuts(self) -> AllSweepCuts:
        count = C.c_uint32(0)
        self._call(self._L.pxr_read_sweep_cuts, None, None, 0, C.byref(count))
        k = int(count.value)
        labels = np.zeros(k, dtype=np.int32)
        cuts = np.zeros(k, dtype=SWEEP_CUT)
        self._call(self._L.pxr_read_sweep_cuts, _ptr(labels), _ptr(cuts), k, C.byref(count))
        return AllSweepCuts(labels, cuts)

    def downloadPartition(self) -> np.ndarray:
        count = C.c_uint32(0)
        self._call(self._L.pxr_download_partition, None, 0, C.byref(count))
        out = np.zeros(int(count.value), dtype=NODE_DATA)
        self._call(self._L.pxr_download_partition, _ptr(out), out.shape[0], C.byref(count))
        return out

    def getFinalPartition(self, out: np.ndarray | None = None) -> FinalPartition:
        """Cluster id of every vertex.  ``out``: an int32 array of n entries
        to write into (page-locked memory makes the device-to-host copy a
        direct DMA; a fresh pageable array is allocated otherwise)."""
        if out is None:
            ids = np.zeros(self.n, dtype=np.int32)
        else:
            if out.dtype != np.int32 or out.shape != (self.n,) or not out.flags.c_contiguous:
                raise ValueError("out must be a contiguous int32 array of n entries")
            ids = out
        k = C.c_int32(0)
        self._call(self._L.pxr_final_partition, _ptr(ids), C.byref(k))
        return FinalPartition(ids, int(k.value))

    def getNumCutEdges(self) -> int:
        out = C.c_uint64(0)
        self._call(self._L.pxr_num_cut_edges, C.byref(out))
        return int(out.value)

    def downloadGraph(self):
        offsets = np.zeros(self.n + 1, dtype=np.uint64)
        cols = np.zeros(2 * self.m, dtype=np.uint32)
        self._call(self._L.pxr_download_graph64, _ptr(offsets), _ptr(cols))
        return offsets, cols

    def downloadDegrees(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=np.uint32)
        self._call(self._L.pxr_download_degrees, _ptr(out))
        return out

    def downloadLabels(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=np.int32)
        self._call(self._L.pxr_download_labels, _ptr(out))
        return out

    def downloadActiveEdgeMap(self) -> np.ndarray:
        out = np.zeros(2 * self.m, dtype=np.int32)
        self._call(self._L.pxr_active_edge_map, _ptr(out))
        return out

    def countCutEdges(self) -> int:
        """Edges whose ends carry different final ids, recounted on the device
        (pxr_count_cut_edges): what the reference's main.cpp computes on the
        host after getFinalPartition (main.cpp:54-60)."""
        out = C.c_uint64(0)
        self._call(self._L.pxr_count_cut_edges, C.byref(out))
        return int(out.value)

    def downloadCertificates(self) -> np.ndarray:
        """Certificate record per vertex (pxr_download_certificates): 0 while
        active, else the certificate's round + 1, bit 31 set when the certified
        set is not the whole set swept that round."""
        out = np.zeros(self.n, dtype=np.uint32)
        self._call(self._L.pxr_download_certificates, _ptr(out))
        return out

    def getNumClusters(self) -> int:
        out = C.c_uint32(0)
        self._call(self._L.pxr_num_active_clusters, C.byref(out))
        return int(out.value)

    def updateLabels(self, nodeLabels=None, activeClusters=None) -> None:
        """No-op, as GraphManager::updateLabels is in the reference."""

    # -- extras -----------------------------------------------------------
    def initialize_device(self, n: int, m: int, offsets_ptr: int, offsets_are_64bit: bool, cols_ptr: int) -> None:
        """initialize() from a CSR already in device memory (raw device pointers)."""
        self._call(self._L.pxr_initialize_device, n, m, C.c_void_p(offsets_ptr), 1 if offsets_are_64bit else 0,
                   C.c_void_p(cols_ptr))
        self.n, self.m = n, m

    def set_profiling(self, enable: bool) -> None:
        self._call(self._L.pxr_set_profiling, 1 if enable else 0)

    def phase_stats(self) -> list[dict]:
        count = C.c_uint32(0)
        self._call(self._L.pxr_phase_stats, None, 0, C.byref(count))
        arr = (_lib.PhaseStat * count.value)()
        self._call(self._L.pxr_phase_stats, arr, count.value, C.byref(count))
        return [{"name": a.name.decode(), "ms": a.ms, "launches": a.launches} for a in arr]

    def stats(self) -> dict:
        st = _lib.Stats()
        self._call(self._L.pxr_get_stats, C.byref(st))
        return {f: getattr(st, f) for f, _ in _lib.Stats._fields_}

    def set_schedule(self, mode: int, weights=None, norm=None, safety: float = 0.5, max_skip: int = 16,
                     trace: bool = False, cut_gate: float = 0.0, due_period: int = 0) -> None:
        """Learned sweep schedule (pxr_set_schedule).  weights: MLP_PARAMS bf16
        bit patterns (uint16); norm: 16 means then 16 scales.  cut_gate: after
        a round that cut more than this fraction of its clusters, the next
        round sweeps every cluster (0: off).  due_period > 1: clusters under
        1/1024 of the active vertices come due only in rounds whose index is
        a multiple of it."""
        cfg = _lib.Schedule(mode, 1 if trace else 0, safety, max_skip, cut_gate, due_period)
        w = n = None
        if weights is not None:
            w = np.ascontiguousarray(weights, dtype=np.uint16)
            assert w.shape[0] == _lib.MLP_PARAMS
            n = np.ascontiguousarray(norm, dtype=np.float32)
            assert n.shape[0] == 2 * _lib.MLP_FEATURES
        self._call(self._L.pxr_set_schedule, C.byref(cfg), _ptr(w) if w is not None else None,
                   _ptr(n) if n is not None else None)

    def cluster_records(self) -> np.ndarray:
        """pxr_cluster_record of every active cluster after the last round (trace mode)."""
        cnt = C.c_uint32(0)
        self._call(self._L.pxr_read_cluster_records, None, 0, C.byref(cnt))
        out = np.zeros(cnt.value, dtype=_lib.RECORD_DTYPE)
        if cnt.value:
            self._call(self._L.pxr_read_cluster_records, _ptr(out), cnt.value, C.byref(cnt))
        return out

    def row_plan(self) -> dict:
        """The row plan in use (pxr_get_row_plan)."""
        rp = _lib.RowPlan()
        self._call(self._L.pxr_get_row_plan, C.byref(rp))
        return {f: getattr(rp, f) for f, _ in _lib.RowPlan._fields_}

    def set_row_plan(self, lanes_per_row: int | None = None, light_max: int = 64, wide_max: int = 4096) -> None:
        """Force a row plan; with no arguments return to the configured tuning."""
        if lanes_per_row is None:
            self._call(self._L.pxr_set_row_plan, None)
            return
        rp = _lib.RowPlan(lanes_per_row, light_max, wide_max)
        self._call(self._L.pxr_set_row_plan, C.byref(rp))

    def sort_plan(self) -> dict:
        """The sweep sort's plan in use (pxr_get_sort_plan)."""
        sp = _lib.SortPlan()
        self._call(self._L.pxr_get_sort_plan, C.byref(sp))
        out = {f: getattr(sp, f) for f, _ in _lib.SortPlan._fields_ if f != "sort_us"}
        out["sort_us"] = [float(v) for v in sp.sort_us]
        return out

    def set_sort_plan(self, plan: int | None = None) -> None:
        """Force sort plan 0, 1 or 2; with no argument return to the configured tuning."""
        if plan is None:
            self._call(self._L.pxr_set_sort_plan, None)
            return
        sp = _lib.SortPlan()
        sp.plan = plan
        self._call(self._L.pxr_set_sort_plan, C.byref(sp))

    def set_stream(self, stream_ptr: int | None) -> None:
        self._call(self._L.pxr_set_stream, C.c_void_p(stream_ptr) if stream_ptr else None)

    def set_potentials(self, x) -> None:
        x = np.ascontiguousarray(x, dtype=np.float64)
        self._call(self._L.pxr_set_potentials, _ptr(x))

    def set_state(self, labels, act, x, ideg, cols, n_clusters, smallest, full_components=True) -> None:
        labels = np.ascontiguousarray(labels, dtype=np.int32)
        act = np.ascontiguousarray(act, dtype=np.uint32)
        x = np.ascontiguousarray(x, dtype=np.float64)
        ideg = np.ascontiguousarray(ideg, dtype=np.uint32)
        cols = np.ascontiguousarray(cols, dtype=np.uint32)
        self._call(self._L.pxr_set_state, _ptr(labels), _ptr(act), act.shape[0], _ptr(x), _ptr(ideg),
                   _ptr(cols), int(n_clusters), int(smallest), 1 if full_components else 0)
