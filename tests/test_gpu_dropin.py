"""Drop-in check: the reference's own application (main.cpp, compiled
unchanged) linked against the CudaDeviceManager shim and libparex_b200.so.
It reads a Matrix Market graph, decomposes it on the GPU and recounts the
cut edges on the CPU (main.cpp:38-60); its printed cluster count and cut
edges must equal what the Python binding reports for the same graph and
seed."""
import os
import re
import subprocess

import numpy as np
import pytest

import parex_b200 as P
from parex_b200 import graphs as G

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BINARY = os.path.join(ROOT, "parex_b200", "cxx", "_build", "parex_main")


@pytest.mark.skipif(not os.path.exists(BINARY), reason="drop-in binary is built where the reference tree exists")
@pytest.mark.parametrize("seed", [6582, 7])
def test_reference_main_runs_on_the_drop_in(tmp_path, seed):
    g = G.sbm_graph()
    path = tmp_path / "sbm16k.mtx"
    G.write_mtx(path, g)
    out = subprocess.run([BINARY, str(path), str(seed), "0.3", "1e-4"], check=True, capture_output=True,
                         text=True, timeout=300).stdout
    fields = dict(re.findall(r"^(\w+): (\S+)$", out, flags=re.M))
    dm = P.CudaDeviceManager(seed=seed)
    dm.initialize(g)
    rounds = dm.expanderDecomposition()
    fp = dm.getFinalPartition()
    src = np.repeat(np.arange(g.n), np.diff(g.offsets.astype(np.int64)))
    recount = int(np.sum(fp.clusterIds[src] != fp.clusterIds[g.cols]) // 2)
    assert int(fields["numClusters"]) == fp.numClusters
    assert int(fields["cutEdges"]) == recount
    assert int(fields["nodes"]) == g.n and int(fields["edges"]) == g.m
    assert int(fields["iterations"]) == rounds
