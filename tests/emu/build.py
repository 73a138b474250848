"""Builds the CPU emulation harness (tests/emu/libmvbt_emu.so) with g++."""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
LIB = HERE / "libmvbt_emu.so"
SRCS = [HERE / "emu.cpp", ROOT / "mvgpubtree_b200" / "csrc" / "validate.cpp"]
DEPS = SRCS + [ROOT / "include" / "mvbt_device.cuh", ROOT / "include" / "mvbt.h"]


def build(force: bool = False) -> Path:
    if not force and LIB.exists() and all(LIB.stat().st_mtime >= d.stat().st_mtime for d in DEPS):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run(["g++", "-std=c++20", "-O1", "-g", "-shared", "-fPIC", f"-I{ROOT / 'include'}",
                    *map(str, SRCS), "-o", str(tmp), "-lpthread"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
