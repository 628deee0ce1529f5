"""Builds the CUDA library libising_b200.so in-tree for sm_100a with nvcc."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "_lib")
LIB_PATH = os.path.join(LIB_DIR, "libising_b200.so")
SOURCES = ["ie_kernels.cu", "ie_level.cu", "ie_level_host.cu", "ie_engine.cu", "ie_static.cu", "ie_v2.cu",
           "ie_pa.cu", "ie_presolve.cu", "ie_local.cu"]
HEADERS = ["ie_device.cuh", "ie_kernels.cuh", "ie_sweep.cuh", "ie_level.cuh", "ie_level_host.h", "ie_launch.h",
           "ie_host.h",
           os.path.join("..", "..", "include", "ising_b200.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared", "-lpthread",
]


def _stale() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    for f in SOURCES + HEADERS:
        if os.path.getmtime(os.path.join(CSRC, f)) > t:
            return True
    return False


def build(force: bool = False) -> str:
    """Compiles the library if it is missing or older than its sources."""
    if not force and not _stale():
        return LIB_PATH
    os.makedirs(LIB_DIR, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *NVCC_FLAGS, "-o", LIB_PATH] + [os.path.join(CSRC, s) for s in SOURCES]
    subprocess.run(cmd, check=True)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force=True))
