"""Failure paths, made on the host or on scratch flags - no GPU fault:

* both bounded device-side waits (the scans' decoupled look-back and the
  sort's tile-status wait) give up on a flag that nothing sets, set their
  error bits and return; the library reports PXR_DEVICE_FAULT as a timed-out
  round does, and the handle decomposes correctly afterwards;
* a handle whose memory cap (pxr_config.memory_cap_mib) is below what a graph
  needs refuses the initialisation with PXR_OUT_OF_MEMORY, keeps nothing, and
  works again for a graph that fits;
* invalid arguments are refused before any device work.
"""
import ctypes as C

import numpy as np
import pytest

import parex_b200 as P
from oracle import oracle as O
from parex_b200 import _lib, graphs as G

pytestmark = pytest.mark.gpu

DEVICE_FAULT, OUT_OF_MEMORY, INVALID_ARG = 5, 2, 1


def _oracle_ids(g, x0):
    orc = O.Oracle(g.offsets, g.cols, O.MODE_PXR)
    orc.set_potentials(x0.astype(np.float64))
    orc.decompose()
    return orc.final_partition()[0]


def test_bounded_waits_time_out_and_handle_stays_usable():
    L = _lib.load()
    g = G.sbm_graph(2048, 8, 10.0, 0.5, 7)
    dm = P.CudaDeviceManager()
    dm.initialize(g)
    bits = C.c_uint32(0)
    assert L.pxr_test_bounded_waits(dm._h, 64, C.byref(bits)) == DEVICE_FAULT
    assert bits.value & 1 and bits.value & 8          # kErrLookback, kErrSortTiles
    assert b"bounded wait" in L.pxr_last_error(dm._h)
    assert L.pxr_test_bounded_waits(dm._h, 0, C.byref(bits)) == INVALID_ARG
    # the same handle still decomposes, bit-exact against the oracle
    dm.initialize(g)
    x0 = dm.readRandomWalkValues()
    dm.expanderDecomposition()
    np.testing.assert_array_equal(dm.getFinalPartition().clusterIds, _oracle_ids(g, x0))


def test_memory_cap_refuses_and_recovers():
    big = G.grid3d(64)
    capped = P.CudaDeviceManager(memory_cap_mib=4)
    with pytest.raises(_lib.PxrError) as info:
        capped.initialize(big)
    assert info.value.status == OUT_OF_MEMORY
    assert capped.stats()["device_bytes"] == 0
    small = G.grid3d(8)
    capped.initialize(small)                           # fits under the cap
    x0 = capped.readRandomWalkValues()
    capped.expanderDecomposition()
    np.testing.assert_array_equal(capped.getFinalPartition().clusterIds, _oracle_ids(small, x0))
    assert 0 < capped.stats()["device_bytes"] <= 4 << 20


def test_invalid_graphs_are_refused():
    dm = P.CudaDeviceManager()
    bad_off = np.array([0, 2, 1, 4], dtype=np.uint32)  # decreasing offsets
    with pytest.raises(_lib.PxrError) as info:
        dm.initialize((bad_off, np.array([1, 2, 0, 0], dtype=np.uint32)))
    assert info.value.status == INVALID_ARG
    out_of_range = np.array([0, 1, 2], dtype=np.uint32)
    with pytest.raises(_lib.PxrError):
        dm.initialize((out_of_range, np.array([1, 5], dtype=np.uint32)))
