"""Builds workload/libworkload.so: the host-only synthetic workload generator (g++, no CUDA).

The generator is harness code shared by the benchmark, the tests and the reference driver
(oracle/ref_driver.cu links the same source). It is kept out of libmvbt.so so that a process that
only generates inputs -- the reference arm of bench.py, the oracle's CPU baseline -- never maps the
product library. Run as ``python workload/build.py [--force]`` (a standalone script).
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "workload.cpp"
HDR = HERE / "mvbt_workload.h"
LIB = HERE / "libworkload.so"


def build(force: bool = False, verbose: bool = False) -> Path:
    deps = [SRC, HDR, Path(__file__)]
    if not force and LIB.exists() and all(d.stat().st_mtime <= LIB.stat().st_mtime for d in deps):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = ["g++", "-std=c++17", "-O3", "-fPIC", "-shared", f"-I{HERE}", str(SRC), "-o", str(tmp), "-lpthread"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
