import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libparex_b200.so")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def golden():
    """Fixtures recorded from the reference's own binaries (tests/golden/make_golden.py)."""
    import json

    def trace(name):
        return dict(np.load(os.path.join(GOLDEN, f"ref_trace_{name}.npz")))

    with open(os.path.join(GOLDEN, "reference_summary.json")) as f:
        summary = json.load(f)
    return {"trace": trace, "summary": summary}


def unpack_valid(bits, cols):
    """Rebuild the CSR column array from a validity bitmask."""
    valid = np.unpackbits(bits)[: cols.shape[0]].astype(bool)
    out = cols.copy()
    out[~valid] = 0xFFFFFFFF
    return out
