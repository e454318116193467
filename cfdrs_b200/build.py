"""In-tree build of libcfdgpu.so (nvcc, sm_100a only) via csrc/Makefile."""
from __future__ import annotations

import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 4) -> str:
    subprocess.run(["make", "-s", f"-j{jobs}", "-C", os.path.join(_HERE, "csrc")], check=True)
    return os.path.join(_HERE, "libcfdgpu.so")


if __name__ == "__main__":
    print(build())
