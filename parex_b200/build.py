"""Build the in-tree CUDA library (nvcc, sm_100a) and the drop-in C++ shim."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 2) -> str:
    subprocess.run(["make", "-s", f"-j{jobs}", "-C", os.path.join(HERE, "csrc")], check=True)
    return os.path.join(HERE, "libparex_b200.so")


if __name__ == "__main__":
    print(build())
