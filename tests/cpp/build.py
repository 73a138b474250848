"""Builds the C++ callers of the library used by the tests: tests/cpp/drop_in_example (a host
caller of include/gpu_btree.h, g++) and tests/cpp/libuser_kernels.so (user kernels written against
include/gpu_btree_device.cuh, nvcc for sm_100a)."""
from __future__ import annotations

import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
EXE = HERE / "drop_in_example"
USER_SO = HERE / "libuser_kernels.so"


def build() -> Path:
    cuda = Path("/usr/local/cuda")
    subprocess.run(["g++", "-std=c++17", "-O2", f"-I{ROOT / 'include'}", f"-I{cuda / 'include'}",
                    str(HERE / "drop_in_example.cpp"), "-o", str(EXE),
                    f"-L{ROOT / 'mvgpubtree_b200'}", "-lmvbt", "-Wl,-rpath,$ORIGIN/../../mvgpubtree_b200",
                    f"-L{cuda / 'lib64'}", "-lcudart"], check=True)
    return EXE


def build_user_kernels(force: bool = False) -> Path:
    src = HERE / "user_kernels.cu"
    deps = [src, Path(__file__)] + sorted((ROOT / "include").glob("*"))
    if not force and USER_SO.exists() and all(d.stat().st_mtime <= USER_SO.stat().st_mtime for d in deps):
        return USER_SO
    cuda = Path("/usr/local/cuda")
    nvcc = str(cuda / "bin" / "nvcc")
    tmp = USER_SO.with_suffix(".so.tmp")
    subprocess.run([nvcc, "-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-Xcompiler", "-fPIC", "-shared", f"-I{ROOT / 'include'}", str(src), "-o", str(tmp),
                    f"-L{ROOT / 'mvgpubtree_b200'}", "-lmvbt", "-Xlinker", "-rpath,$ORIGIN/../../mvgpubtree_b200"],
                   check=True)
    tmp.replace(USER_SO)
    return USER_SO


if __name__ == "__main__":
    print(build())
    print(build_user_kernels(force=True))
