"""GPU tier: the sorted batch front-end of the bulk calls against the oracle and against the
unsorted path.

With MVBT_FRONTEND_SORTED a bulk call sorts its keys on the device (mvbt_sort.cu) and each tile
runs a contiguous run of them, every op starting from the deepest node of the previous op's path
that covers its key. Results must be identical to the oracle's for inserts (a repeated key's last
occurrence wins), updates after a snapshot, erases, and finds and range queries at snapshots, in
both tree kinds and both tile widths, from an empty tree (the growth phase spreads its first
inserts) and on a populated one.
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


def _ranges(torch, t, lo, hi, cap, ts):
    import mvgpubtree_b200 as mv
    n = lo.size
    pairs = torch.full((n * cap * 2,), -1, dtype=torch.int32, device="cuda")
    counts = torch.zeros(n, dtype=torch.int32, device="cuda")
    kw = {"timestamp": ts} if isinstance(t, mv.gpu_versioned_btree) else {}
    t.range_query(dev(torch, lo), dev(torch, hi), pairs, counts, cap, **kw)
    return host(pairs).reshape(n, cap, 2), host(counts)


@pytest.mark.parametrize("frontend", [1, 2])
@pytest.mark.parametrize("w", [8, 16])
def test_frontends_match_oracle_on_versioned_tree(torch, frontend, w):
    import mvgpubtree_b200 as mv
    import oracle
    import workload as wl
    seed, n0 = 41, 1 << 18
    keys = wl.distinct_keys(seed, 0, n0)
    vals = wl.values_for(keys, seed)
    t = mv.gpu_versioned_btree(pool_bytes=1 << 30, tile_width=w, frontend=frontend)
    m = oracle.MVMap(True)
    if frontend == mv.FRONTEND_SORTED:  # repeated keys: the last occurrence wins
        rng = np.random.default_rng(seed)
        dup = rng.choice(n0, 4096, replace=False)
        ik = np.concatenate([keys, keys[dup]])
        iv = np.concatenate([vals, wl.values_for(keys[dup], seed ^ 9)])
    else:
        ik, iv = keys, vals
    t.insert(dev(torch, ik), dev(torch, iv))
    m.insert(ik, iv)
    s0 = t.take_snapshot(); assert s0 == m.take_snapshot()
    upd = wl.shuffle(seed + 1, keys)[: n0 // 4]
    t.insert(dev(torch, upd), dev(torch, wl.values_for(upd, seed ^ 1)))
    m.insert(upd, wl.values_for(upd, seed ^ 1))
    er = wl.shuffle(seed + 2, keys)[: n0 // 5]
    t.erase(dev(torch, er))
    m.erase(er)
    new = wl.distinct_keys(seed, n0, n0 // 3)
    t.insert(dev(torch, new), dev(torch, wl.values_for(new, seed)))
    m.insert(new, wl.values_for(new, seed))
    assert t.check_errors() == 0
    s1 = t.take_snapshot(); assert s1 == m.take_snapshot()
    q = wl.shuffle(seed + 3, np.concatenate([keys, new, wl.distinct_keys(seed, wl.MISS_INDEX_BASE, n0 // 2)]))
    lo = wl.uniform_keys(seed + 4, 1 << 16)
    hi = wl.upper_bounds(lo, 24, wl.stride_for(n0))
    for ts in (s0, s1, mv.LATEST):
        for concurrent in (False, True):
            out = torch.empty(q.size, dtype=torch.int32, device="cuda")
            t.find(dev(torch, q), out, timestamp=ts, concurrent=concurrent)
            assert np.array_equal(host(out), m.find(q, ts)), (ts, concurrent)
        gp, gc = _ranges(torch, t, lo, hi, 64, ts)
        ep, ec = m.range_query(lo, hi, 64, ts)
        assert np.array_equal(gc, ec), ts
        mask = np.arange(64)[None, :] < np.minimum(ec, 64)[:, None]
        assert np.array_equal(gp[mask], ep[mask]), ts
    rep = t.validate_tree_structure()
    assert rep["violations"] == 0 and rep["locked_nodes"] == 0 and rep["keys"] == m.size()
    assert t.check_errors() == 0


@pytest.mark.parametrize("w", [8, 16])
def test_sorted_frontend_on_plain_tree_matches_oracle(torch, w):
    import mvgpubtree_b200 as mv
    import oracle
    import workload as wl
    seed, n0 = 43, 1 << 19
    keys = wl.distinct_keys(seed, 0, n0)
    vals = wl.values_for(keys, seed)
    t = mv.gpu_blink_tree(pool_bytes=1 << 30, tile_width=w, frontend=mv.FRONTEND_SORTED)
    m = oracle.MVMap(False)
    t.insert(dev(torch, keys), dev(torch, vals)); m.insert(keys, vals)
    er = wl.shuffle(seed + 1, keys)[: n0 // 3]
    t.erase(dev(torch, er)); m.erase(er)
    q = wl.shuffle(seed + 2, np.concatenate([keys, wl.distinct_keys(seed, wl.MISS_INDEX_BASE, n0)]))
    out = torch.empty(q.size, dtype=torch.int32, device="cuda")
    t.find(dev(torch, q), out)
    assert np.array_equal(host(out), m.find(q))
    lo = wl.uniform_keys(seed + 3, 1 << 15)
    hi = wl.upper_bounds(lo, 8, wl.stride_for(n0))
    gp, gc = _ranges(torch, t, lo, hi, 32, mv.LATEST)
    ep, ec = m.range_query(lo, hi, 32)
    assert np.array_equal(gc, ec)
    mask = np.arange(32)[None, :] < np.minimum(ec, 32)[:, None]
    assert np.array_equal(gp[mask], ep[mask])
    rep = t.validate_tree_structure()
    assert rep["violations"] == 0 and rep["keys"] == m.size()


def test_sorted_insert_of_4M_keys_into_an_empty_tree(torch):
    """The growth phase (evenly spread inserts while the tree has fewer leaves than the grid has
    tiles) followed by contiguous sorted runs: every key present with its value, structure valid."""
    import mvgpubtree_b200 as mv
    import oracle
    import workload as wl
    seed, n = 47, 1 << 22
    keys = wl.distinct_keys(seed, 0, n)
    vals = wl.values_for(keys, seed)
    t = mv.gpu_versioned_btree(pool_bytes=2 << 30, frontend=mv.FRONTEND_SORTED)
    t.insert(dev(torch, keys), dev(torch, vals))
    q = wl.shuffle(seed, np.concatenate([keys, wl.distinct_keys(seed, wl.MISS_INDEX_BASE, n // 4)]))
    out = torch.empty(q.size, dtype=torch.int32, device="cuda")
    t.find(dev(torch, q), out)
    assert np.array_equal(host(out), oracle.SortedSnapshot(keys, vals).find(q))
    rep = t.validate_tree_structure()
    assert rep["violations"] == 0 and rep["locked_nodes"] == 0 and rep["keys"] == n + 1
    assert t.check_errors() == 0


def test_auto_frontend_gives_the_same_results_as_both(torch):
    import mvgpubtree_b200 as mv
    import workload as wl
    seed, n0 = 53, 1 << 17
    keys = wl.distinct_keys(seed, 0, n0)
    vals = wl.values_for(keys, seed)
    outs = []
    for fe in (mv.FRONTEND_AUTO, mv.FRONTEND_UNSORTED, mv.FRONTEND_SORTED):
        t = mv.gpu_versioned_btree(pool_bytes=1 << 28, frontend=fe)
        t.insert(dev(torch, keys), dev(torch, vals))
        t.set_frontend(fe)
        q = wl.shuffle(seed, np.concatenate([keys, wl.distinct_keys(seed, wl.MISS_INDEX_BASE, n0)]))
        out = torch.empty(q.size, dtype=torch.int32, device="cuda")
        t.find(dev(torch, q), out)
        outs.append(host(out))
        assert t.check_errors() == 0
        t.close()
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[1], outs[2])


@pytest.mark.parametrize("kind", ["versioned", "blink"])
def test_insert_into_a_pristine_tree_is_a_bulk_load_with_the_same_contents(torch, kind):
    """A large insert into a tree nothing has written yet is built bottom up from the sorted call:
    the same contents as the pairs upserted in order (repeated keys: the last occurrence wins; key 0
    replaces the tombstone's value), a valid structure, snapshots and later writes behaving as on
    an insert-built tree."""
    import mvgpubtree_b200 as mv
    import oracle
    import workload as wl
    seed, n0 = 59, 1 << 20
    keys = wl.distinct_keys(seed, 0, n0)
    vals = wl.values_for(keys, seed)
    rng = np.random.default_rng(seed)
    dup = rng.choice(n0, 5000, replace=False)
    ik = np.concatenate([keys, keys[dup], np.array([0, 0xFFFFFFFF], np.uint32)])
    iv = np.concatenate([vals, wl.values_for(keys[dup], seed ^ 3), np.array([77, 5], np.uint32)])
    perm = rng.permutation(ik.size)
    ik, iv = ik[perm], iv[perm]
    cls = mv.gpu_versioned_btree if kind == "versioned" else mv.gpu_blink_tree
    t = cls(pool_bytes=1 << 30)
    m = oracle.MVMap(kind == "versioned")
    t.insert(dev(torch, ik), dev(torch, iv))
    m.insert(ik[ik != 0xFFFFFFFF], iv[ik != 0xFFFFFFFF])
    assert t.check_errors() == 0
    rep = t.validate_tree_structure()
    assert rep["violations"] == 0 and rep["locked_nodes"] == 0 and rep["keys"] == m.size()
    k_all, v_all = m.dump()
    q = np.concatenate([k_all, wl.distinct_keys(seed, wl.MISS_INDEX_BASE, 1 << 16)])
    out = torch.empty(q.size, dtype=torch.int32, device="cuda")
    t.find(dev(torch, q), out)
    assert np.array_equal(host(out), m.find(q))
    if kind == "versioned":  # a snapshot, then updates, erases and inserts on the loaded tree
        s0 = t.take_snapshot(); assert s0 == m.take_snapshot()
        upd = wl.shuffle(seed + 1, keys)[: n0 // 8]
        t.insert(dev(torch, upd), dev(torch, wl.values_for(upd, seed ^ 1))); m.insert(upd, wl.values_for(upd, seed ^ 1))
        er = wl.shuffle(seed + 2, keys)[: n0 // 8]
        t.erase(dev(torch, er)); m.erase(er)
        new = wl.distinct_keys(seed, n0, n0 // 4)
        t.insert(dev(torch, new), dev(torch, wl.values_for(new, seed))); m.insert(new, wl.values_for(new, seed))
        s1 = t.take_snapshot(); assert s1 == m.take_snapshot()
        q2 = np.concatenate([q, new])
        for ts in (s0, s1):
            out2 = torch.empty(q2.size, dtype=torch.int32, device="cuda")
            t.find(dev(torch, q2), out2, timestamp=ts)
            assert np.array_equal(host(out2), m.find(q2, ts)), ts
        rep = t.validate_tree_structure()
        assert rep["violations"] == 0 and rep["keys"] == m.size()
    assert t.check_errors() == 0


def test_bulk_load_reports_a_pool_too_small_and_leaves_the_tree_empty(torch):
    import mvgpubtree_b200 as mv
    import workload as wl
    n = 1 << 20  # needs ~116K nodes; the pool holds 8192
    keys = wl.distinct_keys(61, 0, n)
    t = mv.gpu_versioned_btree(pool_bytes=1 << 20)
    t.insert(dev(torch, keys), dev(torch, wl.values_for(keys, 61)))
    bits = t.check_errors(raise_on_error=False)
    assert bits & 1  # MVBT_DEVERR_POOL_EXHAUSTED
    assert t.stats()["error_sites"].get(17, 0) == 1
    t.clear_errors()
    rep = t.validate_tree_structure()
    assert rep["violations"] == 0 and rep["keys"] == 1  # the tombstone only
