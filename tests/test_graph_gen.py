"""The host C R-MAT builder (oracle/graph_gen.c, used to hand the
benchmark's graph to the reference's CPU decomposition without loading the
product library) builds the same CSR as the numpy generator
(parex_b200.graphs.rmat), which the GPU tests pin against the device
generator (tests/test_gpu_build.py)."""
import numpy as np
import pytest

from oracle import oracle as O
from parex_b200 import graphs as G


@pytest.mark.parametrize("scale,seed", [(8, 1), (12, 3), (15, 7)])
def test_host_rmat_equals_numpy_rmat(scale, seed):
    g = G.rmat(scale, 16, seed=seed)
    off, cols = O.rmat_csr(scale, 16, seed=seed)
    np.testing.assert_array_equal(off.astype(np.int64), g.offsets.astype(np.int64))
    np.testing.assert_array_equal(cols, g.cols)


def test_host_rmat_other_quadrants():
    g = G.rmat(11, 8, a=0.45, b=0.15, c=0.15, seed=9)
    off, cols = O.rmat_csr(11, 8, a=0.45, b=0.15, c=0.15, seed=9)
    np.testing.assert_array_equal(off.astype(np.int64), g.offsets.astype(np.int64))
    np.testing.assert_array_equal(cols, g.cols)
