"""Checksums of tree results, as oracle/ref_driver.cu computes them for the reference build, and a
runner for that driver. Test infrastructure: the GPU tests and the benchmark's verification step
compare this library's results with the reference implementation's on identical inputs through
these sums.

With mix(x) = the SplitMix64 finalizer of x + 0x9E3779B97F4A7C15 and i an op's index in its step:
  find  = sum over finds of mix(i << 32 | value)
  count = sum over range queries of mix((i << 32 | count) ^ 0xC3A5C85C97CB3127)
  pairs = sum over range queries and j < min(count, capacity_i) of
          mix(mix((i << 20 | j) ^ 0xB492B66FBE98F273) ^ (key_j << 32 | value_j))
all modulo 2^64.
"""
from __future__ import annotations

import json
import subprocess
from pathlib import Path

import numpy as np

DRIVER = Path(__file__).resolve().parent / "_ref" / "ref_driver"

_U = np.uint64


def mix64(x: np.ndarray) -> np.ndarray:
    x = x.astype(np.uint64) + _U(0x9E3779B97F4A7C15)
    x = (x ^ (x >> _U(30))) * _U(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> _U(27))) * _U(0x94D049BB133111EB)
    return x ^ (x >> _U(31))


def _sum(x: np.ndarray) -> int:
    return int(np.sum(x, dtype=np.uint64)) if x.size else 0


def find_sum(op_index: np.ndarray, values: np.ndarray) -> int:
    i = op_index.astype(np.uint64)
    return _sum(mix64((i << _U(32)) | values.astype(np.uint64)))


def count_sum(op_index: np.ndarray, counts: np.ndarray) -> int:
    i = op_index.astype(np.uint64)
    return _sum(mix64(((i << _U(32)) | counts.astype(np.uint64)) ^ _U(0xC3A5C85C97CB3127)))


def pairs_sum(op_index: np.ndarray, take: np.ndarray, start: np.ndarray, pairs: np.ndarray) -> int:
    """pairs: uint32 array [n_pairs, 2]; query q's pairs are pairs[start[q] : start[q] + take[q]]."""
    take = take.astype(np.int64)
    total = int(take.sum())
    if total == 0:
        return 0
    qi = np.repeat(op_index.astype(np.uint64), take)
    first = np.repeat(np.cumsum(take) - take, take)
    j = (np.arange(total, dtype=np.int64) - first).astype(np.uint64)
    pos = np.repeat(start.astype(np.int64), take) + j.astype(np.int64)
    kv = (pairs[pos, 0].astype(np.uint64) << _U(32)) | pairs[pos, 1].astype(np.uint64)
    return _sum(mix64(mix64(((qi << _U(20)) | j) ^ _U(0xB492B66FBE98F273)) ^ kv))


def step_sums(batches, result: np.ndarray, range_out: np.ndarray) -> list[int]:
    """[find, count, pairs] of one step of mixed batches run through this library (result per op;
    range_out uint32 [n_pairs, 2] with query i's pairs at out_off[i])."""
    t = batches.type
    idx = np.arange(t.size, dtype=np.uint64)
    f, r = t == 0, t == 3
    cnt = result[r]
    take = np.minimum(cnt, batches.range_cap[r])
    return [find_sum(idx[f], result[f]), count_sum(idx[r], cnt),
            pairs_sum(idx[r], take, batches.out_off[r], range_out)]


def run_driver(*args: str, timeout: int = 600) -> dict:
    """Runs the reference build and returns its JSON line."""
    out = subprocess.run([str(DRIVER), *args], capture_output=True, text=True, timeout=timeout)
    if out.returncode != 0:
        raise RuntimeError(f"ref_driver {' '.join(args)} failed ({out.returncode}): {out.stderr[-2000:]}")
    return json.loads(out.stdout.strip().splitlines()[-1])
