"""Builds tests/cpp/drop_in_example (a C++ caller of include/gpu_btree.h) with g++."""
from __future__ import annotations

import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
EXE = HERE / "drop_in_example"


def build() -> Path:
    cuda = Path("/usr/local/cuda")
    subprocess.run(["g++", "-std=c++17", "-O2", f"-I{ROOT / 'include'}", f"-I{cuda / 'include'}",
                    str(HERE / "drop_in_example.cpp"), "-o", str(EXE),
                    f"-L{ROOT / 'mvgpubtree_b200'}", "-lmvbt", "-Wl,-rpath,$ORIGIN/../../mvgpubtree_b200",
                    f"-L{cuda / 'lib64'}", "-lcudart"], check=True)
    return EXE


if __name__ == "__main__":
    print(build())
