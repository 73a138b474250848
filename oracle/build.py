"""Builds the CPU oracle (test infrastructure) into oracle/liboracle.so with g++."""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "oracle.cpp"
LIB = HERE / "liboracle.so"


def build(force: bool = False) -> Path:
    if not force and LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run(["g++", "-std=c++17", "-O2", "-shared", "-fPIC", "-o", str(tmp), str(SRC),
                    "-lpthread"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
