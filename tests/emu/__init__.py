"""ctypes front-end of the CPU emulation harness (the device tree code compiled for the host)."""
from __future__ import annotations

import ctypes

import numpy as np

from .build import LIB, build

_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(str(LIB))
        u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
        vp, u32, u64, i = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int
        sig = {
            "emu_create": (vp, [i, u32, u32, u32, i]),
            "emu_reclaim": (None, [vp, u32]),
            "emu_destroy": (None, [vp]),
            "emu_errors": (u32, [vp]),
            "emu_bump": (u32, [vp]),
            "emu_snapshot": (u32, [vp]),
            "emu_insert": (None, [vp, u32p, u32p, u64, i, i]),
            "emu_erase": (None, [vp, u32p, u64, i, i]),
            "emu_find": (None, [vp, u32p, u32p, u64, u32, i, i, i]),
            "emu_range": (None, [vp, u32p, u32p, vp, vp, u32, u64, u32, i, i, i]),
            "emu_insert_range": (None, [vp, u32p, u32p, u64, u32p, u32p, u64, vp, vp, u32, i, i]),
            "emu_find_erase": (None, [vp, u32p, u32p, u64, u32p, u64, i, i]),
            "emu_sorted_run": (None, [vp, i, u32p, u32p, vp, vp, vp, u32, u64, u32, i, i]),
            "emu_validate": (i, [vp, u32, vp]),
            "emu_stats": (None, [vp, np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")]),
            "emu_batch_run": (None, [vp, u32, np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS"),
                                     u32p, u32p, u32p,
                                     np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS"),
                                     u32p, u32p, vp, i, i, i, i, u32, vp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(_lib, name)
            f.restype = res
            f.argtypes = args
    return _lib


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


class EmuTree:
    """A tree held in host memory, operated on by the device code run as host threads."""

    def __init__(self, versioned: bool, capacity: int = 1 << 16, tiles: int = 4, W: int = 8,
                 spin_limit: int = 0, chunk: int = 8, reclaim: bool = False):
        self.L = lib()
        self.h = self.L.emu_create(int(versioned), capacity, spin_limit, chunk, int(reclaim))
        self.tiles, self.W = tiles, W

    def __del__(self):
        if getattr(self, "h", None):
            self.L.emu_destroy(self.h)
            self.h = None

    @property
    def errors(self) -> int:
        return int(self.L.emu_errors(self.h))

    def stats(self) -> dict:
        v = np.zeros(26, np.uint64)
        self.L.emu_stats(self.h, v)
        return {"cow": int(v[21]), "splits": int(v[1]), "max_hops": int(v[2]), "max_descent": int(v[3]),
                "error_sites": {i: int(v[4 + i]) for i in range(16) if v[4 + i]}, "restarts": int(v[20]),
                "reclaimed": int(v[22]), "free_nodes": int(v[23]), "reused": int(v[24]),
                "log_dropped": int(v[25])}

    def reclaim(self, min_live_snapshot: int = 0xFFFFFFFF):
        self.L.emu_reclaim(self.h, min_live_snapshot & 0xFFFFFFFF)

    @property
    def bump(self) -> int:
        return int(self.L.emu_bump(self.h))

    def snapshot(self) -> int:
        return int(self.L.emu_snapshot(self.h))

    def insert(self, k, v):
        k, v = _u32(k), _u32(v)
        self.L.emu_insert(self.h, k, v, k.size, self.tiles, self.W)

    def erase(self, k):
        k = _u32(k)
        self.L.emu_erase(self.h, k, k.size, self.tiles, self.W)

    def find(self, k, ts=0xFFFFFFFF, quiescent=False):
        k = _u32(k)
        out = np.empty_like(k)
        self.L.emu_find(self.h, k, out, k.size, ts, self.tiles, self.W, int(quiescent))
        return out

    def range(self, lo, hi, avg_len, ts=0xFFFFFFFF, quiescent=False):
        lo, hi = _u32(lo), _u32(hi)
        n = lo.size
        pairs = np.full((n, avg_len, 2), 0xFFFFFFFF, np.uint32)
        counts = np.zeros(n, np.uint32)
        self.L.emu_range(self.h, lo, hi, pairs.ctypes.data, counts.ctypes.data, avg_len, n, ts,
                         self.tiles, self.W, int(quiescent))
        return pairs, counts

    def sorted_run(self, kind: str, keys, arg=None, avg_len: int = 0, ts=0xFFFFFFFF):
        """The sorted front-end's kernels on the emulator: keys are sorted here (a stable sort, so a
        repeated key keeps its input order), each tile runs a contiguous share with its path
        memory, results come back in input order. kind: find | range | insert | erase | qfind | qrange
        (the find and range query of a tree no writer changes meanwhile)."""
        k = _u32(keys)
        order = np.argsort(k, kind="stable").astype(np.uint32)
        sk = np.ascontiguousarray(k[order])
        code = {"find": 0, "range": 1, "insert": 2, "erase": 3, "qfind": 4, "qrange": 5}[kind]
        a = _u32(arg) if arg is not None else None
        out = np.zeros(k.size, np.uint32)
        pairs = np.full((max(1, k.size), max(1, avg_len), 2), 0xFFFFFFFF, np.uint32) if kind in ("range", "qrange") else None
        self.L.emu_sorted_run(self.h, code, sk, order, a.ctypes.data if a is not None else None,
                              out.ctypes.data, pairs.ctypes.data if pairs is not None else None, avg_len,
                              k.size, ts, self.tiles, self.W)
        if kind in ("range", "qrange"):
            return pairs[: k.size], out
        return out

    def find_erase(self, fk, ek):
        fk, ek = _u32(fk), _u32(ek)
        out = np.empty_like(fk)
        self.L.emu_find_erase(self.h, fk, out, fk.size, ek, ek.size, self.tiles, self.W)
        return out

    def insert_range(self, k, v, lo, hi, avg_len):
        k, v, lo, hi = _u32(k), _u32(v), _u32(lo), _u32(hi)
        pairs = np.full((max(1, lo.size), avg_len, 2), 0xFFFFFFFF, np.uint32)
        counts = np.zeros(max(1, lo.size), np.uint32)
        self.L.emu_insert_range(self.h, k, v, k.size, lo, hi, lo.size, pairs.ctypes.data,
                                counts.ctypes.data, avg_len, self.tiles, self.W)
        return pairs[: lo.size], counts[: lo.size]

    def run_batches(self, b, mode: int = 0, reclaim: bool = False, watermark: int = 0xFFFFFFFF,
                    series=None):
        """Runs workload.Batches; returns (result, range_out words). reclaim: reclamation inside the
        persistent run (series: a uint64 array [num_batches, 4] for the memory samples)."""
        result = np.zeros(b.num_ops, np.uint32)
        out = np.full(max(1, b.range_pairs) * 2, 0xFFFFFFFF, np.uint32)
        self.L.emu_batch_run(self.h, b.num_batches, b.batch_off, b.type, b.key, b.arg, b.out_off,
                             b.range_cap, result, out.ctypes.data, mode, self.tiles, self.W,
                             int(reclaim), watermark, series.ctypes.data if series is not None else None)
        return result, out

    def validate(self, ts=0xFFFFFFFF) -> dict:
        import mvgpubtree_b200 as mv
        rep = mv.mvbt_report()
        st = self.L.emu_validate(self.h, ts, ctypes.byref(rep))
        out = {f: getattr(rep, f) for f, _ in mv.mvbt_report._fields_ if not f.startswith("reserved")}
        out["status"] = st
        return out
