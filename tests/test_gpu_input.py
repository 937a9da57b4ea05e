"""The reference's input path on the device: a Matrix Market body tokenised
as readDynGraph reads it (lib/utils/graph_io.h:49-84: a stream of integers,
two per edge, 1-based) and the CSR built as DynamicGraph::finalize builds it
(lib/core/graph.h:147-184: both directions, duplicates and self-loops kept,
rows sorted).  Checked against a numpy restatement of those two functions,
against the reference's own application reading the same file, and by the
decomposition of the graph read either way."""
import os
import re
import subprocess

import numpy as np
import pytest

import parex_b200 as P
from parex_b200 import _lib, gpu_build as B, graphs as G

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BINARY = os.path.join(ROOT, "parex_b200", "cxx", "_build", "parex_main")


def _restated(data: bytes):
    """readDynGraph + DynamicGraph::finalize in numpy: (offsets, cols, n, m)."""
    _, n, m, body = B.mtx_header(data)
    toks = np.array([int(t) for t in re.findall(rb"\d+", data[body:])[: 2 * m]], dtype=np.int64)
    u, v = toks[0::2] - 1, toks[1::2] - 1
    src = np.concatenate([u, v])
    dst = np.concatenate([v, u])
    order = np.lexsort((dst, src))
    cols = dst[order].astype(np.uint32)
    offsets = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(src, minlength=n), out=offsets[1:])
    return offsets, cols, n, m


def _device(path):
    off, cols, n, m = B.read_mtx(path)
    return off.cpu().numpy().astype(np.int64), cols.cpu().numpy().view(np.uint32), n, m


def _messy_file(path):
    rng = np.random.default_rng(3)
    n = 300
    e = rng.integers(1, n + 1, size=(1500, 2))
    e = np.concatenate([e, e[:40], [[7, 7], [9, 9], [9, 9]]])       # duplicates and self-loops
    seps = [b" ", b"  ", b"\t", b" \t "]
    ends = [b"\n", b"\r\n", b"  \n"]
    lines = [b"%%MatrixMarket matrix coordinate pattern symmetric", b"% a comment", b"%another",
             f"{n} {n} {e.shape[0]}".encode()]
    for k, (a, b) in enumerate(e):
        lines.append(str(a).encode() + seps[k % 4] + str(b).encode())
    data = b""
    for k, line in enumerate(lines):
        data += line + ends[k % 3]
    with open(path, "wb") as f:
        f.write(data)
    return data


def test_messy_file_matches_the_restated_reader(tmp_path):
    path = tmp_path / "messy.mtx"
    data = _messy_file(path)
    want = _restated(data)
    got = _device(path)
    assert got[2:] == want[2:]
    np.testing.assert_array_equal(got[0], want[0])
    np.testing.assert_array_equal(got[1], want[1])


def test_generated_graph_round_trip_and_decomposition(tmp_path):
    g = G.sbm_graph()
    path = tmp_path / "sbm16k.mtx"
    G.write_mtx(path, g)
    off, cols, n, m = _device(path)
    np.testing.assert_array_equal(off, g.offsets.astype(np.int64))
    np.testing.assert_array_equal(cols, g.cols)
    a = P.CudaDeviceManager()
    a.initialize(g)
    a.expanderDecomposition()
    offd, colsd, n2, m2 = B.read_mtx(path)
    b = P.CudaDeviceManager()
    b.initialize_device(n2, m2, offd.data_ptr(), False, colsd.data_ptr())
    b.expanderDecomposition()
    np.testing.assert_array_equal(a.getFinalPartition().clusterIds, b.getFinalPartition().clusterIds)


@pytest.mark.skipif(not os.path.exists(BINARY), reason="drop-in binary is built where the reference tree exists")
def test_reference_application_reads_the_same_graph(tmp_path):
    """The reference's main.cpp reads the file with its own readDynGraph and
    finalize (duplicates and self-loops included) and decomposes it through
    the drop-in; the device-read graph must decompose to the same counts."""
    path = tmp_path / "messy.mtx"
    _messy_file(path)
    out = subprocess.run([BINARY, str(path), "6582", "0.3", "1e-4"], check=True, capture_output=True, text=True,
                         timeout=300).stdout
    fields = dict(re.findall(r"^(\w+): (\S+)$", out, flags=re.M))
    off, cols, n, m = B.read_mtx(path)
    dm = P.CudaDeviceManager()
    dm.initialize_device(n, m, off.data_ptr(), False, cols.data_ptr())
    rounds = dm.expanderDecomposition()
    fp = dm.getFinalPartition()
    assert int(fields["nodes"]) == n and int(fields["edges"]) == m
    assert int(fields["numClusters"]) == fp.numClusters
    assert int(fields["iterations"]) == rounds


def test_malformed_bodies_are_refused(tmp_path):
    short = tmp_path / "short.mtx"
    short.write_bytes(b"4 4 3\n1 2\n2 3\n")                 # 4 numbers for 3 edges
    with pytest.raises(_lib.PxrError):
        B.read_mtx(short)
    zero = tmp_path / "zero.mtx"
    zero.write_bytes(b"4 4 2\n0 2\n2 3\n")                  # ids are 1-based
    with pytest.raises(_lib.PxrError):
        B.read_mtx(zero)
    big = tmp_path / "big.mtx"
    big.write_bytes(b"4 4 2\n1 5\n2 3\n")                   # id above n
    with pytest.raises(_lib.PxrError):
        B.read_mtx(big)
