"""Builds the CUDA library libmpm_b200.so in-tree (sm_100a only).

``python -m mpm_3d_b200.build`` or ``build()`` from Python. The library is
written to ``mpm_3d_b200/lib/`` so that it travels with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_DIR = os.path.join(HERE, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libmpm_b200.so")
SOURCES = [os.path.join(HERE, "csrc", "api.cu")]
HEADERS_DIR = os.path.join(HERE, "csrc")

NVCC_FLAGS = [
    "-ccbin", "/usr/bin/g++",
    "-std=c++17",
    "-O3",
    "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC",
    "-shared",
]


def _newest_source_mtime() -> float:
    paths = list(SOURCES) + [os.path.join(ROOT, "include", "mpm_b200.h")]
    for name in os.listdir(HEADERS_DIR):
        paths.append(os.path.join(HEADERS_DIR, name))
    return max(os.path.getmtime(p) for p in paths)


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles the library if it is missing or older than its sources."""
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= _newest_source_mtime():
        return LIB_PATH
    os.makedirs(LIB_DIR, exist_ok=True)
    tmp = LIB_PATH + ".tmp"
    cmd = [nvcc()] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose else []) + SOURCES + ["-o", tmp]
    subprocess.check_call(cmd)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
