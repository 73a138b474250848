"""Builds oracle/_ref/ref_driver: the reference implementation's unmodified headers, compiled for
sm_100a with the reference's own CUDA flags, driven through its public host API by
oracle/ref_driver.cu (this repository's harness) on inputs from this repository's workload
generator (workload/workload.cpp).

The reference is read in place; nothing of it is copied into the repository. The binary is a
build artefact (git-ignored) that travels with the repository to a GPU machine, where the
reference sources are not needed. Run: python oracle/ref_build.py [--force]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
# The reference checkout: --reference DIR, else MVBT_REFERENCE_DIR, else where this build
# environment keeps it read-only. Only this recipe reads it; nothing at run time does.
DEFAULT_REFERENCE = "/root/reference"
OUT = HERE / "_ref"
EXE = OUT / "ref_driver"

# the reference's CUDA flags (its CMakeLists.txt: -maxrregcount=70, extended lambdas, relaxed
# constexpr, C++17), release optimisation, sm_100a
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-maxrregcount=70", "--expt-extended-lambda",
              "--expt-relaxed-constexpr", "-gencode", "arch=compute_100a,code=sm_100a",
              "-Wno-deprecated-gpu-targets"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def reference_dir(path: str | os.PathLike | None = None) -> Path:
    return Path(path or os.environ.get("MVBT_REFERENCE_DIR") or DEFAULT_REFERENCE)


def build(force: bool = False, verbose: bool = False, reference: str | os.PathLike | None = None) -> Path | None:
    """Returns the driver path, or None where the reference sources are absent and no driver was
    built before (a GPU machine only runs the prebuilt binary)."""
    REFERENCE = reference_dir(reference)
    src = HERE / "ref_driver.cu"
    wl = ROOT / "workload" / "workload.cpp"
    if not (REFERENCE / "include" / "gpu_btree.h").exists():
        return EXE if EXE.exists() else None
    deps = [src, wl, ROOT / "workload" / "mvbt_workload.h", Path(__file__)]
    deps += sorted((REFERENCE / "include").glob("*"))
    if not force and EXE.exists() and all(d.stat().st_mtime <= EXE.stat().st_mtime for d in deps):
        return EXE
    OUT.mkdir(exist_ok=True)
    obj = OUT / "workload.o"
    cmds = [
        ["g++", "-std=c++17", "-O3", "-fPIC", f"-I{ROOT / 'workload'}", "-c", str(wl), "-o", str(obj)],
        # only the reference's include directory is on the path: its gpu_btree.h must win
        [_nvcc(), *NVCC_FLAGS, f"-I{REFERENCE / 'include'}", str(src), str(obj), "-o", str(EXE)],
    ]
    for cmd in cmds:
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return EXE


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser(description="build oracle/_ref/ref_driver from the reference headers")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--reference", default=None, help="reference checkout (default: $MVBT_REFERENCE_DIR)")
    a = ap.parse_args()
    print(build(force=a.force, verbose=True, reference=a.reference))
