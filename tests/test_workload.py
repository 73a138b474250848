"""CPU tier: the synthetic workload generator (keys, values, bounds, mixed batches)."""
import numpy as np
import pytest

import workload as wl


def test_distinct_keys_are_distinct_in_domain_and_deterministic():
    a = wl.distinct_keys(3, 0, 1 << 20)
    assert len(np.unique(a)) == a.size
    assert a.min() >= 1 and a.max() <= wl.KEY_DOMAIN_MAX
    assert np.array_equal(a, wl.distinct_keys(3, 0, 1 << 20))
    assert not np.array_equal(a[:100], wl.distinct_keys(4, 0, 100))
    # disjoint index ranges give disjoint key sets
    b = wl.distinct_keys(3, wl.MISS_INDEX_BASE, 1 << 18)
    assert np.intersect1d(a, b).size == 0
    # a window equals the same indices of a longer run
    assert np.array_equal(wl.distinct_keys(3, 1000, 50), a[1000:1050])


def test_keys_look_uniform():
    a = wl.distinct_keys(9, 0, 1 << 20).astype(np.float64) / 2**32
    hist, _ = np.histogram(a, bins=16, range=(0, 1))
    expected = a.size / 16
    assert np.all(np.abs(hist - expected) < 6 * np.sqrt(expected))


def test_values_and_bounds():
    k = np.array([1, 2, 0xFFFFFFFD], np.uint32)
    v = wl.values_for(k, 5)
    assert v.tolist() == [wl.fmix32(int(x) ^ 5) for x in k]
    assert wl.fmix32(0) == 0 and wl.fmix32(1) == 0x514E28B7  # MurmurHash3 fmix32 test values
    up = wl.upper_bounds(np.array([10, 0xFFFFFF00], np.uint32), 8, 107)
    assert up.tolist() == [10 + 856, 0xFFFFFFFF]
    assert wl.stride_for(40_000_000) == 107


def test_uniform_keys_in_domain():
    u = wl.uniform_keys(1, 100000)
    assert u.min() >= 1 and u.max() <= wl.KEY_DOMAIN_MAX


def test_shuffle_is_a_permutation():
    a = np.arange(1000, dtype=np.uint32)
    s = wl.shuffle(2, a)
    assert sorted(s.tolist()) == a.tolist() and not np.array_equal(s, a)


@pytest.mark.parametrize("fixed", [0, 3000])
def test_mix_generator_invariants(fixed):
    seed, n0 = 21, 30000
    g = wl.MixGenerator(seed, n0, stride=wl.stride_for(n0), fixed_batch=fixed, batch_median=4000)
    present = set(wl.distinct_keys(seed, 0, n0).tolist())
    b = g.generate(10)
    assert b.batch_off[0] == 0 and np.all(np.diff(b.batch_off.astype(np.int64)) > 0)
    if fixed:
        assert np.all(np.diff(b.batch_off) == fixed)
    frac = np.bincount(b.type, minlength=4) / b.num_ops
    assert abs(frac[wl.OP_ERASE] - 0.1) < 0.02 and abs(frac[wl.OP_INSERT] - 0.2) < 0.02
    assert abs(frac[wl.OP_FIND] - 0.5) < 0.02 and abs(frac[wl.OP_RANGE] - 0.2) < 0.02
    hits = finds = 0
    for i in range(b.num_batches):
        lo, hi = int(b.batch_off[i]), int(b.batch_off[i + 1])
        t, k, a = b.type[lo:hi], b.key[lo:hi], b.arg[lo:hi]
        er = k[t == wl.OP_ERASE].tolist()
        ins = k[t == wl.OP_INSERT].tolist()
        assert all(x in present for x in er) and len(set(er)) == len(er)
        assert all(x not in present for x in ins) and len(set(ins)) == len(ins)
        assert np.array_equal(a[t == wl.OP_INSERT], wl.values_for(k[t == wl.OP_INSERT], 0))
        f = k[t == wl.OP_FIND].tolist()
        hits += sum(x in present for x in f)
        finds += len(f)
        r = t == wl.OP_RANGE
        assert np.all(a[r] > k[r])
        cap = b.range_cap[lo:hi][r]
        assert np.all(cap % 8 == 0) and np.all(cap >= 16)
        present.difference_update(er)
        present.update(ins)
    assert abs(hits / finds - 0.5) < 0.03
    assert g.present == len(present)
    # range output slots are disjoint and in op order
    r = b.type == wl.OP_RANGE
    off, cap = b.out_off[r].astype(np.int64), b.range_cap[r].astype(np.int64)
    assert np.all(off[1:] == off[:-1] + cap[:-1]) and off[0] == 0
    assert b.range_pairs == int(off[-1] + cap[-1])


def test_lognormal_batch_sizes():
    g = wl.MixGenerator(1, 1000)
    b = g.generate(2000)
    sizes = np.diff(b.batch_off.astype(np.int64))
    assert sizes.min() >= 1024 and sizes.max() <= 4 << 20
    assert 12000 < np.median(sizes) < 21000
