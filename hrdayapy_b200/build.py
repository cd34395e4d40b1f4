"""Builds libhrdaya_b200.so (all CUDA sources under csrc/) for sm_100a.

    python -m hrdayapy_b200.build

The library is written next to this file so that it ships with the source
tree; nothing is installed into site-packages.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "libhrdaya_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def sources():
    return sorted(CSRC.glob("*.cu"))


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    deps = list(CSRC.glob("*")) + [PKG.parent / "include" / "hrdaya_b200.h"]
    return all(p.stat().st_mtime <= t for p in deps if p.exists())


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and up_to_date():
        return LIB
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    flags = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                    "-I", str(PKG.parent / "include"), "--expt-relaxed-constexpr"]
    if os.environ.get("HP_PRECISE_EXP", "0") != "1":
        flags += ["-DHP_FAST_EXP"]
    # the TTP06 kinetics (mono.cu) use the approximate SFU divide / exp / log;
    # every other unit keeps IEEE FP32 division and square root
    fast = {"mono"}
    objs = []
    for src in sources():
        obj = objdir / (src.stem + ".o")
        extra = ["--use_fast_math"] if src.stem in fast else []
        cmd = [nvcc()] + flags + extra + ["-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc()] + ARCH + ["-shared", "-o", str(tmp)] + objs + ["-lcudart"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
