"""In-tree build of the native library and command line.

``build()`` runs ``make`` on megadock_b200/csrc/Makefile, which compiles the
host C++ and the sm_100a kernels (nvcc -gencode arch=compute_100a,code=sm_100a)
into megadock_b200/lib/libmd_b200.so and megadock_b200/bin/megadock-b200.
"""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent


def build(jobs: int | None = None, verbose: bool = False) -> None:
    jobs = jobs or min(8, os.cpu_count() or 1)
    cmd = ["make", "-C", str(PKG / "csrc"), f"-j{jobs}"]
    res = subprocess.run(cmd, capture_output=not verbose, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"native build failed:\n{res.stdout}\n{res.stderr}")
