"""Generates tests/golden/reference_cases.npz: the reference's own known-answer tests as fixtures.

Each case re-creates the inputs of one reference test and stores the outputs that test asserts,
computed here in plain Python (sets and sorted lists, as the reference's std::set /
std::unordered_set validators do), independently of the C++ oracle:

  unittest_btree.cu (test/unittest_btree.cu:77-87 inputs, 138-251 cases), for both trees:
    Validation, FindExist, FindNotExist, EraseAllTest, EraseNoneTest, EraseAllInsertAllTest
  unittest_versioning.cu (test/unittest_versioning.cu:82-95 inputs, 145-376 cases):
    InsertInPlaceValidation / InsertOutOfPlaceValidation, FindExist, FindNotExist,
    RangeQueryTest (two snapshots)
  find_versioned_test.cu (test/find_versioned_test.cu:81-160): batched inserts, one snapshot per
    batch, finds of every key at every snapshot (to_value = 10 * key)
  find_blink_test.cu (test/find_blink_test.cu): batched inserts and finds without snapshots
  test_bulk_build.cu (test/test_bulk_build.cu:40-79): sorted keys 1..N, values 10 * key, a first
    batch then a second batch, full key set checked

Every case is a list of steps replayed by tests/cases.py against the oracle and the GPU tree.
Dense shuffled keys 1..2N (test/find_versioned_test.cu:84-89) use this script's own seeded
shuffle instead of std::shuffle over mt19937, whose output is library-specific.

Run: python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import random
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE / "reference_cases.npz"
SENTINEL = 0xFFFFFFFF

NUM_KEYS = 1024        # --num-keys default of both gtest suites
RQ_LENGTH = 32         # average_range_length_ of unittest_versioning.cu


def u32(a):
    return np.asarray(a, dtype=np.uint32)


class Case:
    def __init__(self, name, kinds):
        self.name = name
        self.kinds = kinds  # tree kinds the case applies to: "blink", "versioned"
        self.steps = []
        self.arrays = {}

    def arr(self, tag, a):
        key = f"{self.name}__{len(self.arrays)}_{tag}"
        self.arrays[key] = u32(a)
        return key

    def insert(self, keys, values, in_place=True):
        self.steps.append({"op": "insert", "keys": self.arr("k", keys),
                           "values": self.arr("v", values), "in_place": in_place})

    def erase(self, keys):
        self.steps.append({"op": "erase", "keys": self.arr("k", keys)})

    def snapshot(self, expect):
        self.steps.append({"op": "snapshot", "expect": int(expect)})

    def find(self, keys, expect, ts="latest"):
        self.steps.append({"op": "find", "keys": self.arr("k", keys),
                           "expect": self.arr("e", expect), "ts": ts})

    def range(self, lo, hi, avg_len, expect_pairs, expect_counts, ts="latest"):
        self.steps.append({"op": "range", "lo": self.arr("lo", lo), "hi": self.arr("hi", hi),
                           "avg_len": int(avg_len), "expect_pairs": self.arr("p", expect_pairs),
                           "expect_counts": self.arr("c", expect_counts), "ts": ts})

    def contents(self, keys, values, ts="latest"):
        self.steps.append({"op": "contents", "keys": self.arr("k", keys),
                           "values": self.arr("v", values), "ts": ts})


def range_expect(key_set_sorted, values_of, lo, hi, avg_len):
    """Pairs written at slot i (unused entries 0xFFFFFFFF) and counts, as validation.hpp:205-264."""
    import bisect
    n = len(lo)
    pairs = np.full((n, avg_len, 2), SENTINEL, np.uint32)
    counts = np.zeros(n, np.uint32)
    for i in range(n):
        j = bisect.bisect_left(key_set_sorted, int(lo[i]))
        c = 0
        while j < len(key_set_sorted) and key_set_sorted[j] < int(hi[i]):
            k = key_set_sorted[j]
            if c < avg_len:
                pairs[i, c] = (k, values_of(k))
            c += 1
            j += 1
        counts[i] = c
    return pairs, counts


def unittest_btree_cases():
    n = NUM_KEYS
    keys = [2 * (i + 1) for i in range(n)]
    values = list(keys)                       # values[i] = keys[i]
    not_exist = [k + 1 for k in keys]
    cases = []
    both = ["blink", "versioned"]

    c = Case("btree_Validation", both)
    c.insert(keys, values)
    c.contents(sorted([0] + keys), [0] + values)  # the root tombstone {0, 0} is part of the tree
    cases.append(c)

    c = Case("btree_FindExist", both)
    c.insert(keys, values)
    c.find(keys, values)
    cases.append(c)

    c = Case("btree_FindNotExist", both)
    c.insert(keys, values)
    c.find(not_exist, [SENTINEL] * n)
    cases.append(c)

    c = Case("btree_EraseAllTest", both)
    c.insert(keys, values)
    c.erase(keys)
    c.find(keys, [SENTINEL] * n)
    cases.append(c)

    c = Case("btree_EraseNoneTest", both)
    c.insert(keys, values)
    c.erase(not_exist)
    c.find(keys, values)
    cases.append(c)

    c = Case("btree_EraseAllInsertAllTest", both)
    c.insert(keys, values)
    c.erase(keys)
    c.find(keys, [SENTINEL] * n)
    c.insert(keys, values)
    c.find(keys, values)
    cases.append(c)
    return cases


def unittest_versioning_cases():
    n = NUM_KEYS
    keys = [2 * (i + 1) for i in range(n)]
    values = list(keys)
    not_exist = [k + 1 for k in keys]
    lower = list(keys)
    upper = [k + 2 * RQ_LENGTH for k in keys]
    first, second = n // 2, n - n // 2
    cases = []
    ver = ["versioned"]

    for in_place, name in ((True, "InsertInPlaceValidation"), (False, "InsertOutOfPlaceValidation")):
        c = Case(f"versioning_{name}", ver)
        c.insert(keys[:first], values[:first], in_place)
        c.snapshot(0)
        c.contents([0] + keys[:first], [0] + values[:first], ts=0)
        c.insert(keys[first:], values[first:], in_place)
        c.contents([0] + keys, [0] + values)
        c.contents([0] + keys[:first], [0] + values[:first], ts=0)
        cases.append(c)

    c = Case("versioning_FindExist", ver)
    c.insert(keys[:first], values[:first], False)
    c.snapshot(0)
    c.find(keys[:first], values[:first], ts=0)
    c.insert(keys[first:], values[first:], False)
    c.find(keys, values)
    cases.append(c)

    c = Case("versioning_FindNotExist", ver)
    c.insert(keys[:first], values[:first], False)
    c.snapshot(0)
    c.find(keys[first:], [SENTINEL] * second, ts=0)
    c.insert(keys[first:], values[first:], False)
    c.find(not_exist, [SENTINEL] * n)
    cases.append(c)

    c = Case("versioning_RangeQueryTest", ver)
    c.insert(keys[:first], values[:first], False)
    c.snapshot(0)
    s0 = sorted(keys[:first])
    p, cnt = range_expect(s0, lambda k: k, lower[:first], upper[:first], RQ_LENGTH)
    c.range(lower[:first], upper[:first], RQ_LENGTH, p, cnt, ts=0)
    c.insert(keys[first:], values[first:], False)
    c.snapshot(1)
    s1 = sorted(keys)
    p, cnt = range_expect(s1, lambda k: k, lower, upper, RQ_LENGTH)
    c.range(lower, upper, RQ_LENGTH, p, cnt, ts=1)
    # the snapshot-0 view is unchanged after the second batch
    p, cnt = range_expect(s0, lambda k: k, lower[:first], upper[:first], RQ_LENGTH)
    c.range(lower[:first], upper[:first], RQ_LENGTH, p, cnt, ts=0)
    cases.append(c)
    return cases


def find_versioned_cases():
    num_keys, batch = 4096, 1024
    rng = random.Random(0)
    dense = list(range(1, 2 * num_keys + 1))
    rng.shuffle(dense)
    keys = dense[:num_keys]                # generate_keys(2N) then resize(N)
    to_value = lambda x: (10 * x) & 0xFFFFFFFF
    c = Case("find_versioned_test", ["versioned"])
    snaps = []
    for b in range(num_keys // batch):
        lo, hi = b * batch, min((b + 1) * batch, num_keys)
        c.insert(keys[lo:hi], [to_value(k) for k in keys[lo:hi]])
        c.snapshot(b)
        snaps.append(hi)
    for b, hi in enumerate(snaps):
        present = set(keys[:hi])
        c.find(keys, [to_value(k) if k in present else SENTINEL for k in keys], ts=b)
    cases = [c]

    c = Case("find_blink_test", ["blink", "versioned"])
    for b in range(num_keys // batch):
        lo, hi = b * batch, min((b + 1) * batch, num_keys)
        c.insert(keys[lo:hi], [to_value(k) for k in keys[lo:hi]])
        present = set(keys[:hi])
        c.find(keys, [to_value(k) if k in present else SENTINEL for k in keys])
    cases.append(c)
    return cases


def bulk_build_cases():
    num_keys, batch = 2048, 1024
    keys = list(range(1, num_keys + 1))
    vals = [10 * k for k in keys]
    c = Case("test_bulk_build", ["blink", "versioned"])
    c.insert(keys[:batch], vals[:batch])
    c.contents([0] + keys[:batch], [0] + vals[:batch])
    c.insert(keys[batch:], vals[batch:])
    c.contents([0] + keys, [0] + vals)
    return [c]


def main():
    cases = unittest_btree_cases() + unittest_versioning_cases() + find_versioned_cases() + bulk_build_cases()
    arrays = {}
    index = []
    for c in cases:
        arrays.update(c.arrays)
        index.append({"name": c.name, "kinds": c.kinds, "steps": c.steps})
    arrays["__index__"] = np.frombuffer(json.dumps(index).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **arrays)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {len(cases)} cases)")


if __name__ == "__main__":
    main()
