"""parex_b200: B200-native random-walk expander decomposition.

A drop-in for the CudaDeviceManager entry point of Parex (cuda/interface.h):
a CSR graph goes in; cluster labels and cut edges come out.  The compute path
is hand-written sm_100a CUDA in ``libparex_b200.so`` behind a C ABI
(include/parex_b200.h); this package is its Python binding.
"""
from .graphs import CSRGraph, csr_from_edges, grid3d, rmat, random_regular, read_pxg, sbm_graph, sbm_batch, write_pxg
from .manager import AllSweepCuts, CudaDeviceManager, FinalPartition
from ._lib import (COMPONENTS_AUTO, COMPONENTS_PLAIN, COMPONENTS_SAMPLED, DIV_IEEE, DIV_REFERENCE, DRIVER_GRAPH,
                   DRIVER_STREAM, TUNE_AUTO, TUNE_HEURISTIC, PxrError)

__all__ = [
    "CSRGraph", "csr_from_edges", "grid3d", "rmat", "random_regular", "read_pxg", "sbm_graph", "sbm_batch",
    "write_pxg", "AllSweepCuts", "CudaDeviceManager", "FinalPartition", "DIV_IEEE", "DIV_REFERENCE",
    "DRIVER_GRAPH", "DRIVER_STREAM", "TUNE_AUTO", "TUNE_HEURISTIC", "PxrError",
    "COMPONENTS_AUTO", "COMPONENTS_PLAIN", "COMPONENTS_SAMPLED",
]
