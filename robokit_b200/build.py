"""Build libb200ik.so in-tree with nvcc for sm_100a.

    python -m robokit_b200.build          # build if sources are newer
    python -m robokit_b200.build --force
"""

from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OUT = os.path.join(PKG, "_lib", "libb200ik.so")

NVCC_FLAGS = [
    "-gencode",
    "arch=compute_100a,code=sm_100a",
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC",
    "-shared",
]


def _sources() -> list:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
                  glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(INCLUDE, "*.h")))


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(s) > t for s in _sources())


UNITS = ["ik_api.cu", "ik_noalloc.cu", "ik_server.cu"]


def build_library(force: bool = False, verbose: bool = False) -> str:
    """Compile every translation unit in parallel (nvcc -c), then link the shared library."""
    if not force and not needs_build():
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    flags = [f for f in NVCC_FLAGS if f != "-shared"]
    objs, procs = [], []
    for u in UNITS:
        obj = os.path.join(os.path.dirname(OUT), u.replace(".cu", ".o"))
        cmd = [nvcc, *flags, f"-I{INCLUDE}", f"-I{CSRC}", "-c", os.path.join(CSRC, u), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((u, subprocess.Popen(cmd)))
        objs.append(obj)
    failed = [u for u, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, f"nvcc {' '.join(failed)}")
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", *objs, "-o", OUT + ".tmp"],
                   check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
