"""Replays the golden reference cases against a driver (the CPU oracle or the GPU tree)."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden" / "reference_cases.npz"
SENTINEL = 0xFFFFFFFF


def load_cases():
    z = np.load(GOLDEN)
    index = json.loads(bytes(z["__index__"]).decode())
    return z, index


def _ts(step):
    return SENTINEL if step.get("ts", "latest") == "latest" else int(step["ts"])


def replay(driver, z, case):
    """Runs every step of `case` on `driver`; raises AssertionError on the first mismatch."""
    for i, s in enumerate(case["steps"]):
        where = f"{case['name']} step {i} ({s['op']})"
        if s["op"] == "insert":
            driver.insert(z[s["keys"]], z[s["values"]], s.get("in_place", True))
        elif s["op"] == "erase":
            driver.erase(z[s["keys"]])
        elif s["op"] == "snapshot":
            got = driver.snapshot()
            assert got == s["expect"], f"{where}: snapshot id {got} != {s['expect']}"
        elif s["op"] == "find":
            got = driver.find(z[s["keys"]], _ts(s))
            exp = z[s["expect"]]
            bad = np.nonzero(got != exp)[0]
            assert bad.size == 0, f"{where}: {bad.size} mismatches, first at {bad[:5]}: {got[bad[:5]]} != {exp[bad[:5]]}"
        elif s["op"] == "range":
            pairs, counts = driver.range(z[s["lo"]], z[s["hi"]], s["avg_len"], _ts(s))
            exp_c = z[s["expect_counts"]]
            assert np.array_equal(counts, exp_c), f"{where}: counts differ"
            exp_p = z[s["expect_pairs"]].reshape(pairs.shape)
            for q in range(len(exp_c)):
                c = min(int(exp_c[q]), s["avg_len"])
                assert np.array_equal(pairs[q, :c], exp_p[q, :c]), f"{where}: pairs of query {q} differ"
        elif s["op"] == "contents":
            k, v = driver.contents(_ts(s), expected=len(z[s["keys"]]))
            assert np.array_equal(k, z[s["keys"]]), f"{where}: key set differs"
            assert np.array_equal(v, z[s["values"]]), f"{where}: values differ"
        else:
            raise ValueError(s["op"])


class OracleDriver:
    def __init__(self, versioned: bool):
        import oracle
        self.m = oracle.MVMap(versioned)

    def insert(self, k, v, in_place=True):
        self.m.insert(k, v)

    def erase(self, k):
        self.m.erase(k)

    def snapshot(self):
        return self.m.take_snapshot()

    def find(self, k, ts):
        return self.m.find(k, ts)

    def range(self, lo, hi, avg_len, ts):
        return self.m.range_query(lo, hi, avg_len, ts)

    def contents(self, ts, expected=None):
        return self.m.dump(ts)


class GpuDriver:
    """Drives a GPU tree through the package's host API with CUDA tensors."""

    def __init__(self, versioned: bool, tile_width: int = 8, pool_bytes: int = 256 << 20):
        import torch
        import mvgpubtree_b200 as mv
        self.torch = torch
        cls = mv.gpu_versioned_btree if versioned else mv.gpu_blink_tree
        self.tree = cls(pool_bytes=pool_bytes, tile_width=tile_width)
        self.versioned = versioned

    def dev(self, a):
        a = np.ascontiguousarray(a, np.uint32)
        return self.torch.from_numpy(a.view(np.int32)).cuda()

    def host(self, t):
        return t.cpu().numpy().view(np.uint32)

    def insert(self, k, v, in_place=True):
        self.tree.insert(self.dev(k), self.dev(v), in_place=in_place)
        self.tree.check_errors()

    def erase(self, k):
        self.tree.erase(self.dev(k))
        self.tree.check_errors()

    def snapshot(self):
        return self.tree.take_snapshot()

    def find(self, k, ts, concurrent=False):
        out = self.torch.empty(len(k), dtype=self.torch.int32, device="cuda")
        self.tree.find(self.dev(k), out, timestamp=ts, concurrent=concurrent)
        self.tree.check_errors()
        return self.host(out)

    def range(self, lo, hi, avg_len, ts, concurrent=False):
        n = len(lo)
        pairs = self.torch.full((n * avg_len * 2,), -1, dtype=self.torch.int32, device="cuda")
        counts = self.torch.zeros(n, dtype=self.torch.int32, device="cuda")
        self.tree.range_query(self.dev(lo), self.dev(hi), pairs, counts, avg_len, timestamp=ts,
                              concurrent=concurrent)
        self.tree.check_errors()
        return self.host(pairs).reshape(n, avg_len, 2), self.host(counts)

    def contents(self, ts, expected=None):
        cap = (expected or 0) + 64
        pairs, counts = self.range(np.array([0], np.uint32), np.array([SENTINEL], np.uint32), cap, ts)
        c = int(counts[0])
        assert c <= cap, "tree holds more keys than expected"
        rep = self.tree.validate_tree_structure(ts)
        assert rep["keys"] == c, f"walk found {rep['keys']} keys, scan found {c}"
        return pairs[0, :c, 0].copy(), pairs[0, :c, 1].copy()


class EmuDriver:
    """The device tree code compiled for the host, W lanes per tile as threads (tests/emu)."""

    def __init__(self, versioned: bool, tile_width: int = 8, tiles: int = 4, capacity: int = 1 << 15):
        from emu import EmuTree
        self.t = EmuTree(versioned, capacity=capacity, tiles=tiles, W=tile_width)

    def _ok(self):
        assert self.t.errors == 0, f"device error bits {self.t.errors}"

    def insert(self, k, v, in_place=True):
        self.t.insert(k, v)
        self._ok()

    def erase(self, k):
        self.t.erase(k)
        self._ok()

    def snapshot(self):
        return self.t.snapshot()

    def find(self, k, ts):
        r = self.t.find(k, ts)
        self._ok()
        return r

    def range(self, lo, hi, avg_len, ts):
        r = self.t.range(lo, hi, avg_len, ts)
        self._ok()
        return r

    def contents(self, ts, expected=None):
        cap = (expected or 0) + 64
        pairs, counts = self.t.range([0], [SENTINEL], cap, ts)
        c = int(counts[0])
        rep = self.t.validate(ts)
        assert rep["status"] == 0 and rep["violations"] == 0, rep
        assert rep["keys"] == c and rep["locked_nodes"] == 0, rep
        return pairs[0, :c, 0].copy(), pairs[0, :c, 1].copy()
