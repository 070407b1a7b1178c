"""Compile the CUDA library ``libtontofock.so`` for sm_100a (in-tree).

    python -m tonto_b200.build

The library is written next to this file so that it travels with the source tree.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libtontofock.so")
PEAK_LIB = os.path.join(HERE, "libtf_peak.so")

SOURCES = ["tontofock.cu", "tf_mlp.cu"]
DEPS = ["tontofock.cu", "tf_mlp.cu", "tf_device.cuh", "tf_warp.cuh", "tf_group.cuh", "rys_tables.inc", "boys_table.inc", "boys2_table.inc",
        os.path.join("..", "..", "include", "tontofock.h"), os.path.join("..", "..", "include", "tontofock_guess.h")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def flags() -> list:
    return ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
            "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-shared"]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(os.path.join(CSRC, d)) <= t for d in DEPS)


def build_peak(force: bool = False) -> str:
    src = os.path.join(CSRC, "fp64_peak.cu")
    if force or not os.path.exists(PEAK_LIB) or os.path.getmtime(src) > os.path.getmtime(PEAK_LIB):
        subprocess.run([nvcc()] + flags() + ["-o", PEAK_LIB, src], check=True, cwd=CSRC)
    return PEAK_LIB


def build(force: bool = False, verbose: bool = False) -> str:
    build_peak(force)
    if not force and up_to_date():
        return LIB
    cmd = [nvcc()] + flags() + ["-o", LIB + ".tmp"] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=CSRC)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
