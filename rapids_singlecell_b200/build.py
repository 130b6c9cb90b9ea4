"""Build the engine's CUDA library in-tree for sm_100a (nvcc cross-compiles; no GPU needed)."""

from __future__ import annotations

import os
import subprocess
from pathlib import Path

CSRC = Path(__file__).resolve().parent / "csrc"


def build(jobs: int | None = None, verbose: bool = False) -> Path:
    jobs = jobs or min(8, os.cpu_count() or 1)
    cmd = ["make", "-C", os.fspath(CSRC), f"-j{jobs}"]
    res = subprocess.run(cmd, capture_output=not verbose, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"CUDA build failed:\n{res.stdout}\n{res.stderr}")
    from ._lib import LIB_PATH

    return LIB_PATH


if __name__ == "__main__":
    print(build(verbose=True))
