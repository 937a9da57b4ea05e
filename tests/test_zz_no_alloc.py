"""pxr_final_partition_static: the final partition for callers that may not
allocate device memory (their memory belongs to a pooling allocator, or they
cannot afford the synchronisation cudaMalloc/cudaFree may cause).

The entry point takes the caller's device arrays and keeps its working
memory in a fixed array inside the library.  This test calls it through the
C ABI twice in a row, on the labels of two different decompositions, and
checks each result against the allocating entry point pxr_final_partition
and against an independent dense rank of the labels (numpy unique): ids and
cluster count must be identical (integer outputs, bit-exact).  It also runs
the largest accepted size (65,536 labels, extremes of the int32 range
included) twice in a row, no labels at all, and checks that sizes above the
fixed limit are refused.

This file is collected last so that, if it fails, a run stopping at the first
failure has already run every other test; it passes alone in a fresh process
as well as after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

import parex_b200 as P
from parex_b200 import _lib
from parex_b200 import graphs as G

pytestmark = pytest.mark.gpu


def _decomposed_labels(graph):
    dm = P.CudaDeviceManager()
    dm.initialize(graph)
    dm.expanderDecomposition()
    labels = dm.downloadLabels()
    expected = dm.getFinalPartition()
    dm.close()
    return labels, expected


def _static_partition(labels_host):
    import torch

    L = _lib.load()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    labels = torch.from_numpy(labels_host).to(dev)
    ids = torch.full((labels_host.shape[0],), -7, dtype=torch.int32, device=dev)
    num = torch.full((1,), -7, dtype=torch.int32, device=dev)
    status = L.pxr_final_partition_static(C.c_void_p(labels.data_ptr()), labels_host.shape[0],
                                          C.c_void_p(ids.data_ptr()), C.c_void_p(num.data_ptr()),
                                          C.c_void_p(stream.cuda_stream))
    assert status == 0, _lib.STATUS.get(status, status)
    torch.cuda.synchronize(dev)
    return ids.cpu().numpy(), int(num.cpu().item())


def test_static_final_partition_matches_allocating_entry_point_twice_in_a_row():
    cases = [G.grid3d(32), G.sbm_graph(2048, 8, 10.0, 0.5, 7)]   # n = 32768, then 2048
    results = [_decomposed_labels(g) for g in cases]
    for labels, expected in results:
        ids, k = _static_partition(labels)
        assert k == expected.numClusters
        np.testing.assert_array_equal(ids, expected.clusterIds)
        want, kw = _dense_rank(labels)
        assert k == kw
        np.testing.assert_array_equal(ids, want)


def _dense_rank(labels):
    """Ids ordered by label value, independently of the library: the
    reference's sort / unique / lower_bound (cuda/devPartition.h:796-822)."""
    uniq, inv = np.unique(labels, return_inverse=True)
    return inv.astype(np.int32), int(uniq.shape[0])


def test_static_final_partition_matches_an_independent_rank():
    rng = np.random.default_rng(3)
    n = _lib.STATIC_SCRATCH_MAX_LABELS        # the largest accepted size: a full array, the last sort tile
    labels = rng.integers(-40000, 40000, n, dtype=np.int32)
    labels[:5] = [-2**31, 2**31 - 1, -1, 0, -2**31]   # extremes of the label range
    for _ in range(2):                                 # twice in a row: the shared array is reused
        ids, k = _static_partition(labels)
        want, kw = _dense_rank(labels)
        assert k == kw
        np.testing.assert_array_equal(ids, want)
        labels = labels[::-1].copy()


def test_static_final_partition_of_no_labels():
    import torch

    L = _lib.load()
    num = torch.full((1,), -7, dtype=torch.int32, device="cuda")
    status = L.pxr_final_partition_static(None, 0, None, C.c_void_p(num.data_ptr()), None)
    assert status == 0
    torch.cuda.synchronize()
    assert int(num.item()) == 0


def test_static_final_partition_refuses_sizes_above_its_limit():
    L = _lib.load()
    n = _lib.STATIC_SCRATCH_MAX_LABELS + 1
    dummy = C.c_void_p(16)   # never dereferenced: the size check comes first
    status = L.pxr_final_partition_static(dummy, n, dummy, dummy, None)
    assert status == 1       # PXR_INVALID_ARG
