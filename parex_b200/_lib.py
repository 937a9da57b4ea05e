"""ctypes loader for libparex_b200.so (the C ABI of include/parex_b200.h).

The library is built in-tree by ``make -C parex_b200/csrc`` (``__graft_entry__.build()``); there is no CPU
fallback, so a missing or unloadable library raises ImportError.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libparex_b200.so")

PXR_OK = 0
STATUS = {0: "PXR_OK", 1: "PXR_INVALID_ARG", 2: "PXR_OUT_OF_MEMORY", 3: "PXR_ITER_CAP",
          4: "PXR_CUDA_ERROR", 5: "PXR_DEVICE_FAULT", 6: "PXR_NOT_INITIALIZED"}
DIV_IEEE = 0
DIV_REFERENCE = 1
DRIVER_GRAPH = 0
DRIVER_STREAM = 1

# every symbol the header declares, in header order
SYMBOLS = [
    "pxr_config_default", "pxr_status_string", "pxr_last_error", "pxr_create", "pxr_destroy",
    "pxr_set_stream", "pxr_initialize", "pxr_initialize64", "pxr_initialize_device", "pxr_walk_step", "pxr_sweep",
    "pxr_cut_clusters", "pxr_decompose", "pxr_read_potentials", "pxr_read_sweep_cuts",
    "pxr_download_partition", "pxr_final_partition", "pxr_num_cut_edges", "pxr_download_graph",
    "pxr_download_graph64", "pxr_download_degrees", "pxr_download_labels", "pxr_active_edge_map",
    "pxr_count_cut_edges", "pxr_download_certificates", "pxr_num_active_clusters", "pxr_get_stats", "pxr_set_profiling", "pxr_phase_stats",
    "pxr_final_partition_static", "pxr_set_potentials", "pxr_set_state", "pxr_initialize_batched",
    "pxr_set_schedule", "pxr_read_cluster_records", "pxr_mlp_forward", "pxr_mlp_scratch_floats", "pxr_mlp_gradient",
    "pxr_mlp_adam_step", "pxr_get_row_plan", "pxr_set_row_plan", "pxr_build_csr_scratch_bytes", "pxr_build_csr",
    "pxr_rmat_edges", "pxr_sbm_edges", "pxr_initialize_batched_device", "pxr_test_bounded_waits",
    "pxr_get_sort_plan", "pxr_set_sort_plan", "pxr_build_csr_finalize", "pxr_parse_mtx_scratch_bytes",
    "pxr_parse_mtx_body", "pxr_contract_scratch_bytes", "pxr_contract",
]
STATIC_SCRATCH_MAX_LABELS = 65536


class SortPlan(C.Structure):
    _fields_ = [("plan", C.c_uint32), ("items_per_thread", C.c_uint32), ("ctas_per_sm", C.c_uint32),
                ("source", C.c_uint32), ("candidates", C.c_uint32), ("sort_us", C.c_float * 3)]


class Config(C.Structure):
    _fields_ = [("seed", C.c_uint32), ("sc_threshold", C.c_float), ("rw_threshold", C.c_float),
                ("max_rounds", C.c_uint32), ("device", C.c_int32), ("division", C.c_uint32),
                ("driver", C.c_uint32), ("tune", C.c_uint32), ("components", C.c_uint32),
                ("memory_cap_mib", C.c_uint32), ("reserved", C.c_uint32 * 6)]


TUNE_AUTO, TUNE_HEURISTIC = 0, 1
COMPONENTS_AUTO, COMPONENTS_PLAIN, COMPONENTS_SAMPLED = 0, 1, 2


class RowPlan(C.Structure):
    _fields_ = [("lanes_per_row", C.c_uint32), ("light_max", C.c_uint32), ("wide_max", C.c_uint32),
                ("wide_rows", C.c_uint32), ("heavy_rows", C.c_uint32), ("source", C.c_uint32),
                ("candidates", C.c_uint32), ("walk_us", C.c_float)]


class SweepCut(C.Structure):
    _fields_ = [("label", C.c_int32), ("sparsity", C.c_float), ("offset", C.c_uint32)]


class NodeData(C.Structure):
    _fields_ = [("nix", C.c_uint32), ("prefix_volume", C.c_uint32), ("prefix_edge_diff", C.c_int32),
                ("offset_in_cluster", C.c_uint32)]


class Stats(C.Structure):
    _fields_ = [("rounds", C.c_uint32), ("active_vertices", C.c_uint32), ("active_clusters", C.c_uint32),
                ("clusters_with_cut", C.c_uint32), ("device_bytes", C.c_uint64),
                ("last_decompose_ms", C.c_double), ("kernel_launches", C.c_uint64),
                ("walk_vertices", C.c_uint64), ("walk_slots", C.c_uint64), ("walk_gathers", C.c_uint64),
                ("sort_items", C.c_uint64), ("sort_passes", C.c_uint64), ("swept_items", C.c_uint64),
                ("skipped_sweeps", C.c_uint64), ("false_stops", C.c_uint64)]


MLP_FEATURES = 16
MLP_HIDDEN = 32
MLP_PARAMS = 1633
SCHEDULE_PLAIN, SCHEDULE_LEARNED, SCHEDULE_AUDIT = 0, 1, 2


class Schedule(C.Structure):
    _fields_ = [("mode", C.c_uint32), ("trace", C.c_uint32), ("safety", C.c_float), ("max_skip", C.c_uint32),
                ("cut_gate", C.c_float), ("due_period", C.c_uint32), ("reserved", C.c_uint32 * 2)]


class ClusterRecord(C.Structure):
    _fields_ = [("root", C.c_uint32), ("size", C.c_uint32), ("volume", C.c_uint32), ("origin", C.c_uint32),
                ("potential", C.c_float), ("sparsity", C.c_float), ("prev_potential", C.c_float),
                ("prev_sparsity", C.c_float), ("prev_round", C.c_uint32), ("age", C.c_uint32),
                ("round", C.c_uint32), ("skip", C.c_uint32), ("prediction", C.c_float), ("has_prev", C.c_uint32),
                ("reserved", C.c_uint32 * 2), ("features", C.c_float * MLP_FEATURES)]


SBM_TASK_DTYPE = np.dtype([("base_u", "<u4"), ("base_v", "<u4"), ("su", "<u4"), ("sv", "<u4"), ("p", "<f8"),
                           ("intra", "<u4"), ("key", "<u4")])


class MlpLoss(C.Structure):
    _fields_ = [("delta", C.c_float), ("over_weight", C.c_float)]


class MlpAdam(C.Structure):
    _fields_ = [("lr", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float)]


RECORD_DTYPE = np.dtype([("root", "<u4"), ("size", "<u4"), ("volume", "<u4"), ("origin", "<u4"),
                         ("potential", "<f4"), ("sparsity", "<f4"), ("prev_potential", "<f4"),
                         ("prev_sparsity", "<f4"), ("prev_round", "<u4"), ("age", "<u4"), ("round", "<u4"),
                         ("skip", "<u4"), ("prediction", "<f4"), ("has_prev", "<u4"), ("reserved", "<u4", 2),
                         ("features", "<f4", MLP_FEATURES)])


class PhaseStat(C.Structure):
    _fields_ = [("name", C.c_char * 24), ("ms", C.c_double), ("launches", C.c_uint64)]


class PxrError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


_lib = None


def load() -> C.CDLL:
    """Load the library (raises ImportError if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; build it with make -C parex_b200/csrc (or __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    p = C.c_void_p
    u32, u64, i32 = C.c_uint32, C.c_uint64, C.c_int32
    L.pxr_config_default.argtypes = [C.POINTER(Config)]
    L.pxr_config_default.restype = None
    L.pxr_status_string.argtypes = [C.c_int]
    L.pxr_status_string.restype = C.c_char_p
    L.pxr_last_error.argtypes = [p]
    L.pxr_last_error.restype = C.c_char_p
    L.pxr_create.argtypes = [C.POINTER(Config), C.POINTER(p)]
    L.pxr_destroy.argtypes = [p]
    L.pxr_destroy.restype = None
    L.pxr_set_stream.argtypes = [p, p]
    L.pxr_initialize.argtypes = [p, u32, u64, p, p]
    L.pxr_initialize64.argtypes = [p, u32, u64, p, p]
    L.pxr_initialize_device.argtypes = [p, u32, u64, p, C.c_int, p]
    L.pxr_set_profiling.argtypes = [p, C.c_int]
    L.pxr_phase_stats.argtypes = [p, C.POINTER(PhaseStat), u32, C.POINTER(u32)]
    for name in ["pxr_walk_step", "pxr_sweep", "pxr_cut_clusters"]:
        getattr(L, name).argtypes = [p]
    L.pxr_decompose.argtypes = [p, C.POINTER(u32)]
    L.pxr_read_potentials.argtypes = [p, p]
    L.pxr_read_sweep_cuts.argtypes = [p, p, p, u32, C.POINTER(u32)]
    L.pxr_download_partition.argtypes = [p, p, u32, C.POINTER(u32)]
    L.pxr_final_partition.argtypes = [p, p, C.POINTER(i32)]
    L.pxr_num_cut_edges.argtypes = [p, C.POINTER(u64)]
    L.pxr_download_graph.argtypes = [p, p, p]
    L.pxr_download_graph64.argtypes = [p, p, p]
    L.pxr_download_degrees.argtypes = [p, p]
    L.pxr_download_labels.argtypes = [p, p]
    L.pxr_active_edge_map.argtypes = [p, p]
    L.pxr_count_cut_edges.argtypes = [p, C.POINTER(u64)]
    L.pxr_test_bounded_waits.argtypes = [p, u32, C.POINTER(u32)]
    L.pxr_get_sort_plan.argtypes = [p, C.POINTER(SortPlan)]
    L.pxr_build_csr_finalize.argtypes = [u32, u64, p, p, p, p, p, p]
    L.pxr_parse_mtx_scratch_bytes.argtypes = [u64]
    L.pxr_parse_mtx_scratch_bytes.restype = C.c_size_t
    L.pxr_parse_mtx_body.argtypes = [p, u64, u32, u64, p, p, p, C.POINTER(u64), p]
    L.pxr_contract_scratch_bytes.argtypes = [u64]
    L.pxr_contract_scratch_bytes.restype = C.c_size_t
    L.pxr_contract.argtypes = [u32, p, p, p, u32, p, p, p, p, C.POINTER(u64), p, p, p]
    L.pxr_set_sort_plan.argtypes = [p, C.POINTER(SortPlan)]
    L.pxr_download_certificates.argtypes = [p, p]
    L.pxr_num_active_clusters.argtypes = [p, C.POINTER(u32)]
    L.pxr_get_stats.argtypes = [p, C.POINTER(Stats)]
    L.pxr_final_partition_static.argtypes = [p, u32, p, p, p]
    L.pxr_set_potentials.argtypes = [p, p]
    L.pxr_set_state.argtypes = [p, p, p, u32, p, p, p, u32, i32, C.c_int]
    L.pxr_initialize_batched.argtypes = [p, u32, u64, p, p, u32, p]
    L.pxr_set_schedule.argtypes = [p, C.POINTER(Schedule), p, p]
    L.pxr_get_row_plan.argtypes = [p, C.POINTER(RowPlan)]
    L.pxr_build_csr_scratch_bytes.argtypes = [u64]
    L.pxr_build_csr.argtypes = [u32, u64, p, p, p, p, p, C.POINTER(u64), p]
    L.pxr_rmat_edges.argtypes = [u32, u64, C.c_double, C.c_double, C.c_double, u64, p, p, p]
    L.pxr_sbm_edges.argtypes = [p, u32, p, u64, u64, u64, p, p, p, p, p]
    L.pxr_initialize_batched_device.argtypes = [p, u32, u64, p, C.c_int, p, u32, p]
    L.pxr_set_row_plan.argtypes = [p, C.POINTER(RowPlan)]
    L.pxr_read_cluster_records.argtypes = [p, p, u32, C.POINTER(u32)]
    L.pxr_mlp_forward.argtypes = [p, u32, p, p, p, p]
    L.pxr_mlp_scratch_floats.argtypes = [u32]
    L.pxr_mlp_gradient.argtypes = [p, p, u32, p, p, C.POINTER(MlpLoss), p, p, p, p]
    L.pxr_mlp_adam_step.argtypes = [p, p, p, p, p, u32, C.POINTER(MlpAdam), p]
    for name in SYMBOLS:
        fn = getattr(L, name)
        if name not in ("pxr_config_default", "pxr_status_string", "pxr_last_error", "pxr_destroy",
                        "pxr_mlp_scratch_floats", "pxr_build_csr_scratch_bytes"):
            fn.restype = C.c_int
    L.pxr_mlp_scratch_floats.restype = C.c_size_t
    L.pxr_build_csr_scratch_bytes.restype = C.c_size_t
    _lib = L
    return L


def check(handle, status: int) -> None:
    if status != PXR_OK:
        L = load()
        msg = L.pxr_last_error(handle).decode() if handle else L.pxr_status_string(status).decode()
        raise PxrError(status, msg)
