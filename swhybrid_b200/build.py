"""In-tree build of libswb200.so for sm_100a (nvcc cross-compiles without a GPU)."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8, verbose: bool = False) -> str:
    cmd = ["make", "-C", os.path.join(HERE, "csrc"), f"-j{jobs}"]
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("libswb200 build failed:\n" + out.stdout[-4000:] + out.stderr[-4000:])
    if verbose:
        print(out.stdout)
    return os.path.join(HERE, "libswb200.so")


if __name__ == "__main__":
    print(build(verbose=True))
