"""CPU oracle (test infrastructure only).

Only tests, the smoke entry point and the benchmark's CPU-baseline leg use this package; it is
the checker, never the thing measured or shipped. It wraps oracle/oracle.cpp (a multiversion
ordered map that restates the reference's validators) through ctypes.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from .build import LIB, build

_lib = None


def _load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = ctypes.CDLL(str(LIB))
        u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
        u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
        vp, u32, u64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64
        sig = {
            "orc_create": (vp, [ctypes.c_int]),
            "orc_destroy": (None, [vp]),
            "orc_current_epoch": (u32, [vp]),
            "orc_take_snapshot": (u32, [vp]),
            "orc_insert": (None, [vp, u32p, u32p, u64]),
            "orc_erase": (None, [vp, u32p, u64]),
            "orc_find": (None, [vp, u32p, u32p, u64, u32]),
            "orc_range": (None, [vp, u32p, u32p, vp, vp, u32, u64, u32]),
            "orc_size": (u64, [vp, u32]),
            "orc_dump": (u64, [vp, u32, vp, vp, u64]),
            "orc_run_batches": (None, [vp, u32, u64p, u32p, u32p, u32p, u64p, u32p, u32p, vp]),
            "orc_part_create": (vp, [ctypes.c_int, u32]),
            "orc_part_destroy": (None, [vp]),
            "orc_part_insert": (None, [vp, u32p, u32p, u64]),
            "orc_part_run_batches": (None, [vp, u32, u64p, u32p, u32p, u32p, u64p, u32p, u32p, vp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(_lib, name)
            f.restype = res
            f.argtypes = args
    return _lib


LATEST = 0xFFFFFFFF
NOT_FOUND = 0xFFFFFFFF


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


class MVMap:
    """Multiversion ordered map: one logical std::map state per snapshot."""

    def __init__(self, versioned: bool = True):
        self._lib = _load()
        self._h = self._lib.orc_create(int(versioned))

    def close(self):
        if getattr(self, "_h", None):
            self._lib.orc_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    @property
    def epoch(self) -> int:
        return int(self._lib.orc_current_epoch(self._h))

    def take_snapshot(self) -> int:
        return int(self._lib.orc_take_snapshot(self._h))

    def insert(self, keys, values):
        k, v = _u32(keys), _u32(values)
        self._lib.orc_insert(self._h, k, v, k.size)

    def erase(self, keys):
        k = _u32(keys)
        self._lib.orc_erase(self._h, k, k.size)

    def find(self, keys, ts: int = LATEST) -> np.ndarray:
        k = _u32(keys)
        out = np.empty_like(k)
        self._lib.orc_find(self._h, k, out, k.size, ts)
        return out

    def range_query(self, lower, upper, avg_len: int, ts: int = LATEST, with_pairs: bool = True):
        """Returns (pairs [n, avg_len, 2] filled with 0xFFFFFFFF past each count, counts [n])."""
        lo, hi = _u32(lower), _u32(upper)
        n = lo.size
        counts = np.zeros(n, np.uint32)
        pairs = np.full((n, avg_len, 2), 0xFFFFFFFF, np.uint32) if with_pairs else None
        self._lib.orc_range(self._h, lo, hi,
                            pairs.ctypes.data if with_pairs else None, counts.ctypes.data,
                            avg_len, n, ts)
        return pairs, counts

    def size(self, ts: int = LATEST) -> int:
        return int(self._lib.orc_size(self._h, ts))

    def dump(self, ts: int = LATEST):
        n = self.size(ts)
        k = np.empty(n, np.uint32)
        v = np.empty(n, np.uint32)
        self._lib.orc_dump(self._h, ts, k.ctypes.data, v.ctypes.data, n)
        return k, v

    def run_batches(self, b, with_pairs: bool = True):
        """Applies mixed batches (workload.Batches); returns (result, range_out)."""
        result = np.zeros(b.num_ops, np.uint32)
        out = np.full(max(1, b.range_pairs) * 2, 0xFFFFFFFF, np.uint32) if with_pairs else None
        self._lib.orc_run_batches(self._h, b.num_batches, b.batch_off, b.type, b.key, b.arg,
                                  b.out_off, b.range_cap, result,
                                  out.ctypes.data if with_pairs else None)
        return result, out


class PartitionedMVMap:
    """Key-range-partitioned oracle: one MVMap per thread (times the CPU baseline on all cores)."""

    def __init__(self, parts: int, versioned: bool = True):
        self._lib = _load()
        self.parts = int(parts)
        self._h = self._lib.orc_part_create(int(versioned), self.parts)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.orc_part_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def insert(self, keys, values):
        k, v = _u32(keys), _u32(values)
        self._lib.orc_part_insert(self._h, k, v, k.size)

    def run_batches(self, b, with_pairs: bool = True):
        result = np.zeros(b.num_ops, np.uint32)
        out = np.full(max(1, b.range_pairs) * 2, 0xFFFFFFFF, np.uint32) if with_pairs else None
        self._lib.orc_part_run_batches(self._h, b.num_batches, b.batch_off, b.type, b.key, b.arg,
                                       b.out_off, b.range_cap, result,
                                       out.ctypes.data if with_pairs else None)
        return result, out


class SortedSnapshot:
    """The oracle's state at one snapshot of a tree that holds exactly `keys` -> `values` (plus the
    tombstone key 0 -> 0 every tree starts with), as sorted arrays. Range queries follow the
    reference's validator (include/validation.hpp:205-238: std::set::lower_bound, then walk while
    key < upper): the hits of [lo, hi) are the keys at sorted positions [lower_bound(lo),
    lower_bound(hi)), ascending. Used where the state is a plain key set (the initial tree of a
    workload) and the queries are too many for the ordered-map oracle's walk: needles are sorted
    before the binary searches, which keeps them cache-friendly."""

    def __init__(self, keys, values):
        k = np.concatenate([np.zeros(1, np.uint32), _u32(keys)])
        v = np.concatenate([np.zeros(1, np.uint32), _u32(values)])
        order = np.argsort(k, kind="stable")
        self.keys, self.values = k[order], v[order]
        if self.keys.size > 1 and not np.all(self.keys[1:] > self.keys[:-1]):
            raise ValueError("SortedSnapshot needs distinct keys")

    def lower_bound(self, q) -> np.ndarray:
        q = _u32(q)
        order = np.argsort(q, kind="stable")
        out = np.empty(q.size, np.int64)
        out[order] = np.searchsorted(self.keys, q[order], side="left")
        return out

    def range_query(self, lower, upper):
        """(start, count): query i's hits are keys[start[i] : start[i] + count[i]] (an empty range
        when upper <= lower, as in validation.hpp)."""
        a = self.lower_bound(lower)
        b = self.lower_bound(upper)
        return a, np.maximum(b - a, 0)

    def find(self, q) -> np.ndarray:
        q = _u32(q)
        pos = np.minimum(self.lower_bound(q), self.keys.size - 1)
        hit = self.keys[pos] == q
        return np.where(hit, self.values[pos], np.uint32(NOT_FOUND)).astype(np.uint32)
