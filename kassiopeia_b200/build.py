"""In-tree build of libkemcu.so for sm_100a (and of the CPU oracles when asked).

    python -m kassiopeia_b200.build          # library only
    python -m kassiopeia_b200.build --all    # library + oracle/ (test infrastructure)
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libkemcu.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "-shared",
]


def _sources():
    return sorted(os.path.join(SRC, f) for f in os.listdir(SRC)
                  if f.endswith((".cu", ".cuh", ".inc")))


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.exists(cand) or cand == "nvcc"):
            return cand
    return "nvcc"


def build_library(force: bool = False, verbose: bool = False) -> str:
    srcs = _sources() + [os.path.join(ROOT, "include", "kemcu.h")]
    if not force and os.path.exists(LIB):
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(s) <= t for s in srcs):
            return LIB
    cmd = [nvcc(), *NVCC_FLAGS, "-I" + os.path.join(ROOT, "include"), "-o", LIB + ".tmp",
           os.path.join(SRC, "kemcu_lib.cu")]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


def build_oracle() -> None:
    """oracle/libkemoracle.so always; oracle/_ref/libkemref.so where the reference tree exists."""
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "-j8", "all"], check=True)


def build(all_parts: bool = True, force: bool = False) -> None:
    build_library(force=force)
    if all_parts:
        build_oracle()


if __name__ == "__main__":
    build(all_parts="--all" in sys.argv, force="--force" in sys.argv)
