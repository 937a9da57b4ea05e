"""ctypes binding of the CPU oracle (test infrastructure: tests, smoke(), bench CPU baseline).

Loads ``oracle/liboracle.so`` built from ``oracle/pxr_oracle.c`` by
``oracle/Makefile``.  Nothing in the ``parex_b200`` package imports this.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

MODE_REF = 0
MODE_PXR = 1

LNODE = np.dtype([("nix", "<u4"), ("label", "<i4")])
NODE_DATA = np.dtype([("nix", "<u4"), ("prefix_volume", "<u4"), ("prefix_edge_diff", "<i4"),
                      ("offset", "<u4")])
SWEEP_CUT = np.dtype([("label", "<i4"), ("sparsity", "<f4"), ("offset", "<u4")])
CLUSTER_DATA = np.dtype([("sum", "<f4"), ("max", "<f4"), ("min", "<f4"), ("count", "<u4")])


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        p = C.c_void_p
        L.orc_create.restype = p
        L.orc_create.argtypes = [C.c_uint32, C.c_uint64, p, p, C.c_int, C.c_float, C.c_float]
        L.orc_destroy.argtypes = [p]
        L.orc_initial_potentials.argtypes = [C.c_uint32, p, C.c_uint32, p]
        L.orc_set_potentials.argtypes = [p, p]
        L.orc_get_potentials.argtypes = [p, p]
        L.orc_set_state.argtypes = [p, p, p, C.c_uint32, p, p, p, C.c_uint32, C.c_int32]
        for name in ["orc_walk", "orc_sweep", "orc_cut_stage", "orc_components_stage",
                     "orc_cluster_data_stage", "orc_recenter_stage", "orc_disable_stage",
                     "orc_cut_clusters", "orc_rekey"]:
            getattr(L, name).argtypes = [p]
        L.orc_scheduled_round.argtypes = [p, p]
        L.orc_decompose.argtypes = [p, C.c_uint32]
        L.orc_decompose.restype = C.c_uint32
        L.orc_final_partition.argtypes = [p, p]
        L.orc_final_partition.restype = C.c_int32
        L.orc_num_cut_edges.argtypes = [p]
        L.orc_num_cut_edges.restype = C.c_uint64
        for name in ["orc_n_active", "orc_n_clusters", "orc_n_sweep_clusters", "orc_n_cuts",
                     "orc_n_data_clusters"]:
            getattr(L, name).argtypes = [p]
            getattr(L, name).restype = C.c_uint32
        L.orc_rmat_csr.argtypes = [C.c_uint32, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, p,
                                   C.POINTER(p), C.POINTER(C.c_uint64)]
        L.orc_rmat_csr.restype = C.c_int
        L.orc_free.argtypes = [p]
        L.orc_smallest_label.argtypes = [p]
        L.orc_smallest_label.restype = C.c_int32
        for name in ["orc_labels", "orc_active", "orc_internal_degrees", "orc_cols", "orc_keys",
                     "orc_sorted", "orc_sweep_labels", "orc_sweep_volumes", "orc_all_cuts",
                     "orc_cuts", "orc_data_labels", "orc_cluster_values", "orc_certificates"]:
            getattr(L, name).argtypes = [p]
            getattr(L, name).restype = p
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _view(addr, dtype, count) -> np.ndarray:
    dtype = np.dtype(dtype)
    if count == 0 or not addr:
        return np.zeros(0, dtype=dtype)
    buf = (C.c_char * (dtype.itemsize * count)).from_address(addr)
    return np.frombuffer(buf, dtype=dtype, count=count).copy()


def initial_potentials(offsets: np.ndarray, seed: int) -> np.ndarray:
    off = np.ascontiguousarray(offsets, dtype=np.uint64)
    n = off.shape[0] - 1
    out = np.zeros(n, dtype=np.float32)
    lib().orc_initial_potentials(n, _ptr(off), seed, _ptr(out))
    return out


def rmat_csr(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
             seed: int = 1):
    """R-MAT CSR (offsets uint64[n+1], cols uint32[2m]) built on the host in C
    (oracle/graph_gen.c): the graph of parex_b200.graphs.rmat and of the
    library's device generator, without loading the library."""
    n = 1 << scale
    ta, tab, tabc = (int(round(t * 65536)) for t in (a, a + b, a + b + c))
    off = np.zeros(n + 1, dtype=np.uint64)
    cols_p = C.c_void_p()
    m = C.c_uint64(0)
    if lib().orc_rmat_csr(scale, edge_factor << scale, ta, tab, tabc, seed, _ptr(off), C.byref(cols_p),
                          C.byref(m)) != 0:
        raise MemoryError("orc_rmat_csr: out of host memory")
    try:
        cols = np.ctypeslib.as_array((C.c_uint32 * (2 * m.value)).from_address(cols_p.value)).copy() \
            if m.value else np.zeros(0, dtype=np.uint32)
    finally:
        lib().orc_free(cols_p)
    return off, cols


class Oracle:
    """One decomposition state in the oracle; methods mirror the round's stages."""

    def __init__(self, offsets, cols, mode=MODE_PXR, sc_threshold=0.3, rw_threshold=1e-4):
        self.off = np.ascontiguousarray(offsets, dtype=np.uint64)
        self.cols0 = np.ascontiguousarray(cols, dtype=np.uint32)
        self.n = self.off.shape[0] - 1
        self.m = self.cols0.shape[0] // 2
        self.mode = mode
        self._s = lib().orc_create(self.n, self.m, _ptr(self.off), _ptr(self.cols0), mode,
                                   sc_threshold, rw_threshold)

    def __del__(self):
        if getattr(self, "_s", None):
            lib().orc_destroy(self._s)
            self._s = None

    # state
    def set_potentials(self, x) -> None:
        x = np.ascontiguousarray(x, dtype=np.float64)
        lib().orc_set_potentials(self._s, _ptr(x))

    def potentials(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=np.float64)
        lib().orc_get_potentials(self._s, _ptr(out))
        return out

    def set_state(self, labels, act, x, ideg, cols, n_clusters, smallest) -> None:
        labels = np.ascontiguousarray(labels, dtype=np.int32)
        act = np.ascontiguousarray(act, dtype=LNODE)
        x = np.ascontiguousarray(x, dtype=np.float64)
        ideg = np.ascontiguousarray(ideg, dtype=np.uint32)
        cols = np.ascontiguousarray(cols, dtype=np.uint32)
        lib().orc_set_state(self._s, _ptr(labels), _ptr(act), act.shape[0], _ptr(x), _ptr(ideg),
                            _ptr(cols), n_clusters, smallest)

    # stages
    def walk(self): lib().orc_walk(self._s)
    def sweep(self): lib().orc_sweep(self._s)
    def cut_stage(self): lib().orc_cut_stage(self._s)
    def components_stage(self): lib().orc_components_stage(self._s)
    def cluster_data_stage(self): lib().orc_cluster_data_stage(self._s)
    def recenter_stage(self): lib().orc_recenter_stage(self._s)
    def disable_stage(self): lib().orc_disable_stage(self._s)
    def cut_clusters(self): lib().orc_cut_clusters(self._s)
    def rekey(self): lib().orc_rekey(self._s)

    def scheduled_round(self, due) -> None:
        """One round in which only the clusters with due[c] != 0 are swept."""
        due = np.ascontiguousarray(due, dtype=np.uint8)
        assert due.shape[0] >= self.n_clusters
        lib().orc_scheduled_round(self._s, _ptr(due) if due.size else None)

    def decompose(self, max_rounds: int = 200000) -> int:
        return int(lib().orc_decompose(self._s, max_rounds))

    def final_partition(self):
        ids = np.zeros(self.n, dtype=np.int32)
        k = lib().orc_final_partition(self._s, _ptr(ids))
        return ids, int(k)

    def num_cut_edges(self) -> int:
        return int(lib().orc_num_cut_edges(self._s))

    # views
    @property
    def n_active(self): return int(lib().orc_n_active(self._s))
    @property
    def n_clusters(self): return int(lib().orc_n_clusters(self._s))
    @property
    def n_sweep_clusters(self): return int(lib().orc_n_sweep_clusters(self._s))
    @property
    def n_cuts(self): return int(lib().orc_n_cuts(self._s))
    @property
    def n_data_clusters(self): return int(lib().orc_n_data_clusters(self._s))
    @property
    def smallest_label(self): return int(lib().orc_smallest_label(self._s))

    def labels(self): return _view(lib().orc_labels(self._s), np.int32, self.n)
    def active(self): return _view(lib().orc_active(self._s), LNODE, self.n_active)
    def internal_degrees(self): return _view(lib().orc_internal_degrees(self._s), np.uint32, self.n)
    def cols(self): return _view(lib().orc_cols(self._s), np.uint32, 2 * self.m)
    def keys(self, count): return _view(lib().orc_keys(self._s), np.uint64, count)
    def sorted(self): return _view(lib().orc_sorted(self._s), NODE_DATA, self.n_active)
    def sweep_labels(self): return _view(lib().orc_sweep_labels(self._s), np.int32, self.n_sweep_clusters)
    def sweep_volumes(self): return _view(lib().orc_sweep_volumes(self._s), np.uint32, self.n_sweep_clusters)
    def all_cuts(self): return _view(lib().orc_all_cuts(self._s), SWEEP_CUT, self.n_sweep_clusters)
    def cuts(self): return _view(lib().orc_cuts(self._s), SWEEP_CUT, self.n_cuts)
    def data_labels(self): return _view(lib().orc_data_labels(self._s), np.int32, self.n_data_clusters)
    def cluster_values(self): return _view(lib().orc_cluster_values(self._s), CLUSTER_DATA, self.n_data_clusters)
    def certificates(self): return _view(lib().orc_certificates(self._s), np.uint32, self.n).copy()
