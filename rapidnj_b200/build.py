"""Builds the in-tree native artefacts for sm_100a.

* ``rapidnj_b200/librnjgpu.so``  -- the C ABI (nvcc -gencode arch=compute_100a,code=sm_100a)
* the C++ drop-in and CLI objects under ``rapidnj_b200/host`` (when present)
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 4) -> None:
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", os.path.join(HERE, "csrc")], check=True)
    host = os.path.join(HERE, "host")
    if os.path.exists(os.path.join(host, "Makefile")):
        subprocess.run(["make", "-s", "-j", str(jobs), "-C", host], check=True)


if __name__ == "__main__":
    build()
