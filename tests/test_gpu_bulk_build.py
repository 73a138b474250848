"""GPU tier: bulk build from sorted pairs (mvbt_bulk_build), the counterpart of the reference's
bulk-build constructor (include/gpu_blink_tree.hpp:85-136).

The built tree holds exactly the tombstone {0, 0} and the given pairs, passes the structural walk,
and behaves like any tree afterwards (inserts that split full leaves, erases, snapshots), checked
against the oracle; the reference's test_bulk_build.cu flow (sorted keys 1..N with values 10 * key
built, then a second batch inserted) is replayed; unsorted input and used trees are refused.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need CUDA"
    return t


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, np.uint32).view(np.int32)).cuda()


def host(t):
    return t.cpu().numpy().view(np.uint32)


def find(torch, t, keys, ts=0xFFFFFFFF):
    out = torch.empty(len(keys), dtype=torch.int32, device="cuda")
    t.find(dev(torch, keys), out, timestamp=ts)
    return host(out)


@pytest.mark.parametrize("kind", ["blink", "versioned"])
@pytest.mark.parametrize("w,fill", [(8, 8), (16, 13), (8, 2)])
def test_bulk_built_tree_matches_oracle_and_keeps_working(torch, kind, w, fill):
    import workload as wl
    import mvgpubtree_b200 as mv
    import oracle
    seed, n = 5, 200_000 if fill > 2 else 20_000
    keys = np.sort(wl.distinct_keys(seed, 0, n))
    vals = wl.values_for(keys, seed)
    cls = mv.gpu_versioned_btree if kind == "versioned" else mv.gpu_blink_tree
    t = cls(pool_bytes=1 << 28, tile_width=w)
    t.bulk_build(dev(torch, keys), dev(torch, vals), fill=fill)
    rep = t.validate_tree_structure()
    assert rep["violations"] == 0 and rep["keys"] == n + 1
    m = oracle.MVMap(kind == "versioned")
    m.insert(keys, vals)
    q = np.concatenate([keys, wl.distinct_keys(seed, wl.MISS_INDEX_BASE, 5000), np.array([0], np.uint32)])
    assert np.array_equal(find(torch, t, q), m.find(q))
    lo = wl.uniform_keys(seed, 2000)
    hi = wl.upper_bounds(lo, 32, wl.stride_for(n))
    pairs = torch.full((2000 * 64 * 2,), -1, dtype=torch.int32, device="cuda")
    counts = torch.empty(2000, dtype=torch.int32, device="cuda")
    t.range_query(dev(torch, lo), dev(torch, hi), pairs, counts, 64, 2000)
    ep, ec = m.range_query(lo, hi, 64, 0xFFFFFFFF)
    assert np.array_equal(host(counts), ec)
    gp = host(pairs).reshape(2000, 64, 2)
    mask = np.arange(64)[None, :] < np.minimum(ec, 64)[:, None]
    assert np.array_equal(gp[mask], ep[mask])
    # afterwards: a snapshot, inserts (splitting full leaves), updates and erases
    s0 = None
    if kind == "versioned":
        s0 = t.take_snapshot()
        assert s0 == m.take_snapshot()
    more = wl.distinct_keys(seed, n, n // 4)
    upd = wl.shuffle(seed + 1, keys)[: n // 8]
    er = wl.shuffle(seed + 2, keys)[: n // 8]
    t.insert(dev(torch, more), dev(torch, wl.values_for(more, 3)))
    t.insert(dev(torch, upd), dev(torch, wl.values_for(upd, 4)))
    t.erase(dev(torch, er))
    m.insert(more, wl.values_for(more, 3))
    m.insert(upd, wl.values_for(upd, 4))
    m.erase(er)
    assert t.check_errors() == 0
    q2 = np.concatenate([q, more])
    assert np.array_equal(find(torch, t, q2), m.find(q2))
    if s0 is not None:
        assert np.array_equal(find(torch, t, q, s0), m.find(q, s0))
    assert t.validate_tree_structure()["violations"] == 0


def test_reference_bulk_build_flow_and_key_zero(torch):
    """test/test_bulk_build.cu: sorted keys 1..N with values 10 * key built, the full set checked,
    then a second batch inserted and the full set checked again; a key 0 in the input replaces
    the tombstone's value."""
    import mvgpubtree_b200 as mv
    N, batch = 2048, 1024
    keys = np.arange(1, N + 1, dtype=np.uint32)
    vals = keys * 10
    t = mv.gpu_blink_tree(pool_bytes=1 << 24)
    t.bulk_build(dev(torch, keys[:batch]), dev(torch, vals[:batch]))
    assert np.array_equal(find(torch, t, np.concatenate([[0], keys[:batch]])), np.concatenate([[0], vals[:batch]]))
    assert np.all(find(torch, t, keys[batch:]) == 0xFFFFFFFF)
    t.insert(dev(torch, keys[batch:]), dev(torch, vals[batch:]))
    assert np.array_equal(find(torch, t, keys), vals)
    assert t.validate_tree_structure()["keys"] == N + 1
    z = mv.gpu_versioned_btree(pool_bytes=1 << 24)
    z.bulk_build(dev(torch, np.array([0, 5, 9], np.uint32)), dev(torch, np.array([77, 50, 90], np.uint32)))
    assert list(find(torch, z, np.array([0, 5, 9, 7], np.uint32))) == [77, 50, 90, 0xFFFFFFFF]


def test_bulk_build_refuses_unsorted_input_and_used_trees(torch):
    import mvgpubtree_b200 as mv
    t = mv.gpu_blink_tree(pool_bytes=1 << 24)
    with pytest.raises(mv.MVBTError):
        t.bulk_build(dev(torch, np.array([3, 2, 5], np.uint32)), dev(torch, np.array([1, 1, 1], np.uint32)))
    with pytest.raises(mv.MVBTError):
        t.bulk_build(dev(torch, np.array([2, 2, 5], np.uint32)), dev(torch, np.array([1, 1, 1], np.uint32)))
    with pytest.raises(mv.MVBTError):
        t.bulk_build(dev(torch, np.array([1, 0xFFFFFFFF], np.uint32)), dev(torch, np.array([1, 1], np.uint32)))
    t.insert(dev(torch, np.array([4], np.uint32)), dev(torch, np.array([4], np.uint32)))
    with pytest.raises(mv.MVBTError):
        t.bulk_build(dev(torch, np.array([1, 2], np.uint32)), dev(torch, np.array([1, 1], np.uint32)))
    v = mv.gpu_versioned_btree(pool_bytes=1 << 24)
    v.take_snapshot()
    with pytest.raises(mv.MVBTError):
        v.bulk_build(dev(torch, np.array([1, 2], np.uint32)), dev(torch, np.array([1, 1], np.uint32)))
