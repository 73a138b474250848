"""GPU tier: the sm_100a tree against the oracle and the reference's known answers (bit-exact).

Every call goes through the C ABI of libmvbt.so (via the package's ctypes mirror).
"""
import numpy as np
import pytest

from cases import GpuDriver, OracleDriver, load_cases, replay

pytestmark = pytest.mark.gpu

SENT = 0xFFFFFFFF


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need CUDA"
    return t


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, np.uint32).view(np.int32)).cuda()


def host(t):
    return t.cpu().numpy().view(np.uint32)


def _case_params():
    _, index = load_cases()
    return [pytest.param(c["name"], kind, w, id=f"{c['name']}-{kind}-w{w}")
            for c in index for kind in c["kinds"] for w in (8, 16)]


@pytest.mark.parametrize("name,kind,w", _case_params())
def test_reference_known_answers(torch, name, kind, w):
    z, index = load_cases()
    case = next(c for c in index if c["name"] == name)
    replay(GpuDriver(kind == "versioned", tile_width=w), z, case)


@pytest.mark.parametrize("w", [8, 16])
@pytest.mark.parametrize("n", [1 << 12, 1 << 20])
def test_plain_tree_insert_find_matches_oracle(torch, w, n):
    """Plain B-link tree, n distinct uniform keys, n shuffled finds (half hits, half misses)."""
    import workload as wl
    import mvgpubtree_b200 as mv
    import oracle
    seed = 1234
    keys = wl.distinct_keys(seed, 0, n)
    vals = wl.values_for(keys, seed)
    hits = wl.shuffle(seed + 1, keys)[: n // 2]
    miss = wl.distinct_keys(seed, wl.MISS_INDEX_BASE, n - n // 2)
    q = wl.shuffle(seed + 2, np.concatenate([hits, miss]))
    t = mv.gpu_blink_tree(pool_bytes=1 << 30, tile_width=w)
    t.insert(dev(torch, keys), dev(torch, vals))
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    t.find(dev(torch, q), out)
    assert t.check_errors() == 0
    m = oracle.MVMap(False)
    m.insert(keys, vals)
    assert np.array_equal(host(out), m.find(q))
    rep = t.validate_tree_structure()
    assert rep["keys"] == n + 1 and rep["locked_nodes"] == 0 and rep["violations"] == 0


@pytest.mark.parametrize("w", [8, 16])
def test_versioned_updates_snapshots_match_oracle(torch, w):
    """Versioned tree: build, S0, update a subset, S1, finds at S0 and S1 (50 % hits)."""
    import workload as wl
    import mvgpubtree_b200 as mv
    import oracle
    seed, n, nu = 77, 1 << 18, 1 << 15
    keys = wl.distinct_keys(seed, 0, n)
    vals = wl.values_for(keys, seed)
    upd = wl.shuffle(seed + 5, keys)[:nu]
    uval = wl.values_for(upd, seed ^ 1)
    q = wl.shuffle(seed + 6, np.concatenate([wl.shuffle(seed + 7, keys)[: n // 2],
                                              wl.distinct_keys(seed, wl.MISS_INDEX_BASE, n // 2)]))
    t = mv.gpu_versioned_btree(pool_bytes=1 << 30, tile_width=w)
    m = oracle.MVMap(True)
    t.insert(dev(torch, keys), dev(torch, vals)); m.insert(keys, vals)
    s0 = t.take_snapshot(); assert s0 == m.take_snapshot()
    t.insert(dev(torch, upd), dev(torch, uval)); m.insert(upd, uval)
    s1 = t.take_snapshot(); assert s1 == m.take_snapshot()
    for ts in (s0, s1, mv.LATEST):
        out = torch.empty(n, dtype=torch.int32, device="cuda")
        t.find(dev(torch, q), out, timestamp=ts)
        assert np.array_equal(host(out), m.find(q, ts)), f"ts={ts}"
    assert t.check_errors() == 0
    for ts in (s0, s1):
        rep = t.validate_tree_structure(ts)
        assert rep["violations"] == 0 and rep["keys"] == n + 1


def _range_check(t, m, torch, lo, hi, cap, ts, concurrent=False):
    n = len(lo)
    pairs = torch.full((n * cap * 2,), -1, dtype=torch.int32, device="cuda")
    counts = torch.zeros(n, dtype=torch.int32, device="cuda")
    t.range_query(dev(torch, lo), dev(torch, hi), pairs, counts, cap, timestamp=ts, concurrent=concurrent)
    assert t.check_errors() == 0
    ep, ec = m.range_query(lo, hi, cap, ts)
    gp = host(pairs).reshape(n, cap, 2)
    gc = host(counts)
    assert np.array_equal(gc, ec)
    written = np.minimum(ec, cap)
    mask = np.arange(cap)[None, :] < written[:, None]
    assert np.array_equal(gp[mask], ep[mask])
    assert np.all(gp[~mask] == SENT), "pairs written past the count"


@pytest.mark.parametrize("w", [8, 16])
@pytest.mark.parametrize("L", [8, 32, 128])
def test_range_queries_at_snapshots_match_oracle(torch, w, L):
    import workload as wl
    import mvgpubtree_b200 as mv
    import oracle
    seed, n, nq = 99, 1 << 17, 1 << 14
    stride = wl.stride_for(n)
    keys = wl.distinct_keys(seed, 0, n)
    t = mv.gpu_versioned_btree(pool_bytes=1 << 30, tile_width=w)
    m = oracle.MVMap(True)
    t.insert(dev(torch, keys), dev(torch, wl.values_for(keys, seed)))
    m.insert(keys, wl.values_for(keys, seed))
    s0 = t.take_snapshot(); m.take_snapshot()
    more = wl.distinct_keys(seed, n, n // 2)
    t.insert(dev(torch, more), dev(torch, wl.values_for(more, seed)))
    m.insert(more, wl.values_for(more, seed))
    er = wl.shuffle(seed + 3, keys)[: n // 4]
    t.erase(dev(torch, er)); m.erase(er)
    lo = wl.uniform_keys(seed + 9, nq)
    hi = wl.upper_bounds(lo, L, stride)
    cap = ((L + 6 * int(np.sqrt(L)) + 16 + 7) // 8) * 8
    for ts in (s0, mv.LATEST):
        _range_check(t, m, torch, lo, hi, cap, ts)


@pytest.mark.parametrize("w", [8, 16])
@pytest.mark.parametrize("u", [0.05, 0.5, 0.9])
def test_concurrent_insert_range_matches_oracle(torch, w, u):
    """One kernel of inserts + range queries; queries read the snapshot taken at launch."""
    import workload as wl
    import mvgpubtree_b200 as mv
    import oracle
    seed, n0, nops, L = 5, 1 << 18, 1 << 16, 32
    stride = wl.stride_for(n0)
    keys = wl.distinct_keys(seed, 0, n0)
    t = mv.gpu_versioned_btree(pool_bytes=1 << 30, tile_width=w)
    m = oracle.MVMap(True)
    t.insert(dev(torch, keys), dev(torch, wl.values_for(keys, seed)))
    m.insert(keys, wl.values_for(keys, seed))
    rng = np.random.default_rng(seed)
    n_ins = int((rng.random(nops) < u).sum())
    n_rq = nops - n_ins
    ins = wl.distinct_keys(seed, n0, n_ins)
    lo = wl.uniform_keys(seed + 1, n_rq)
    hi = wl.upper_bounds(lo, L, stride)
    cap = 96
    pairs = torch.full((max(1, n_rq) * cap * 2,), -1, dtype=torch.int32, device="cuda")
    counts = torch.zeros(max(1, n_rq), dtype=torch.int32, device="cuda")
    t.concurrent_insert_range(dev(torch, ins), dev(torch, wl.values_for(ins, seed)), n_ins,
                              dev(torch, lo), dev(torch, hi), n_rq, pairs, cap, counts)
    assert t.check_errors() == 0
    s = m.take_snapshot()
    ep, ec = m.range_query(lo, hi, cap, s)
    m.insert(ins, wl.values_for(ins, seed))
    gc = host(counts)[:n_rq]
    assert np.array_equal(gc, ec)
    gp = host(pairs)[: n_rq * cap * 2].reshape(n_rq, cap, 2)
    mask = np.arange(cap)[None, :] < np.minimum(ec, cap)[:, None]
    assert np.array_equal(gp[mask], ep[mask])
    # every insert landed
    out = torch.empty(n_ins, dtype=torch.int32, device="cuda")
    t.find(dev(torch, ins), out)
    assert np.array_equal(host(out), wl.values_for(ins, seed))
    assert t.validate_tree_structure()["keys"] == n0 + n_ins + 1


@pytest.mark.parametrize("kind", ["versioned", "blink"])
def test_concurrent_find_erase(torch, kind):
    import workload as wl
    import mvgpubtree_b200 as mv
    import oracle
    seed, n0 = 8, 1 << 17
    keys = wl.distinct_keys(seed, 0, n0)
    vals = wl.values_for(keys, seed)
    cls = mv.gpu_versioned_btree if kind == "versioned" else mv.gpu_blink_tree
    t = cls(pool_bytes=1 << 30)
    t.insert(dev(torch, keys), dev(torch, vals))
    before = torch.empty(n0, dtype=torch.int32, device="cuda")
    t.find(dev(torch, keys), before)
    assert np.array_equal(host(before), vals), "tree wrong before the concurrent phase"
    er = wl.shuffle(seed + 1, keys)[: n0 // 2]
    fk = wl.shuffle(seed + 2, keys)[: n0 // 2]
    out = torch.empty(len(fk), dtype=torch.int32, device="cuda")
    t.concurrent_find_erase(dev(torch, fk), out, len(fk), dev(torch, er), len(er))
    assert t.check_errors() == 0
    got = host(out)
    expect = wl.values_for(fk, seed)
    if kind == "versioned":
        assert np.array_equal(got, expect)  # finds read the launch snapshot
    else:
        # reference acceptance (include/validation.hpp:106-149): found, or the key was erased
        erased = np.isin(fk, er)
        ok = (got == expect) | (erased & (got == SENT))
        bad = np.nonzero(~ok)[0]
        assert bad.size == 0, (
            f"{bad.size} bad finds: {int(np.sum(~erased[bad] & (got[bad] == SENT)))} live keys not "
            f"found, {int(np.sum(got[bad] != SENT))} wrong values; first: "
            + ", ".join(f"key {int(fk[i]):#x} got {int(got[i]):#x} expect {int(expect[i]):#x} "
                        f"erased {bool(erased[i])}" for i in bad[:4])
            + f"; stats {t.stats()}")
    out2 = torch.empty(len(keys), dtype=torch.int32, device="cuda")
    t.find(dev(torch, keys), out2)
    m = oracle.MVMap(kind == "versioned")
    m.insert(keys, vals)
    m.erase(er)
    assert np.array_equal(host(out2), m.find(keys))


@pytest.mark.parametrize("w", [8, 16])
def test_edge_cases(torch, w):
    import mvgpubtree_b200 as mv
    t = mv.gpu_versioned_btree(pool_bytes=1 << 28, tile_width=w)
    z = torch.empty(0, dtype=torch.int32, device="cuda")
    t.insert(z, z); t.find(z, z); t.erase(z)  # empty inputs are no-ops
    out = torch.empty(3, dtype=torch.int32, device="cuda")
    t.find(dev(torch, [0, 1, SENT]), out)
    assert host(out).tolist() == [0, SENT, SENT]  # root tombstone {0, 0}
    t.insert(dev(torch, [SENT, 5, 5]), dev(torch, [1, 7, 7]))  # reserved key ignored, duplicates upsert
    t.find(dev(torch, [SENT, 5]), out[:2])
    assert host(out)[:2].tolist() == [SENT, 7]
    # dense consecutive keys (all into one leaf chain), then descending keys
    asc = np.arange(1000, 3000, dtype=np.uint32)
    t.insert(dev(torch, asc), dev(torch, asc * 3))
    desc = np.arange(9000, 7000, -1, dtype=np.uint32)
    t.insert(dev(torch, desc), dev(torch, desc + 1))
    allk = np.concatenate([asc, desc])
    out = torch.empty(len(allk), dtype=torch.int32, device="cuda")
    t.find(dev(torch, allk), out)
    assert np.array_equal(host(out), np.concatenate([asc * 3, desc + 1]))
    # ranges: empty (lo >= hi), truncated to the slot with the full count, saturated upper bound
    import oracle
    m = oracle.MVMap(True)
    m.insert([5], [7]); m.insert(asc, asc * 3); m.insert(desc, desc + 1)
    _range_check(t, m, torch, np.array([2000, 1000, 8990, 0], np.uint32),
                 np.array([2000, SENT, SENT, 10], np.uint32), 16, mv.LATEST)
    assert t.check_errors() == 0
    rep = t.validate_tree_structure()
    assert rep["violations"] == 0 and rep["locked_nodes"] == 0 and rep["keys"] == 1 + 1 + 2000 + 2000


def test_pool_exhaustion_is_reported_not_hung(torch):
    """A tiny pool: inserts stop with MVBT_ERR_POOL_EXHAUSTED and the tree stays readable."""
    import workload as wl
    import mvgpubtree_b200 as mv
    t = mv.gpu_blink_tree(pool_bytes=1024 * 128, tile_width=8, chunk_nodes=8)
    keys = wl.distinct_keys(3, 0, 1 << 16)
    t.insert(dev(torch, keys), dev(torch, keys))
    bits = t.check_errors(raise_on_error=False)
    assert bits & 1
    with pytest.raises(mv.MVBTError):
        t.check_errors()
    rep = t.validate_tree_structure(raise_on_error=False)
    assert rep["locked_nodes"] == 0
    out = torch.empty(len(keys), dtype=torch.int32, device="cuda")
    t.find(dev(torch, keys), out)
    got = host(out)
    assert np.all((got == keys) | (got == SENT))  # every find returns a stored value or a miss


def test_spin_limit_gives_up_without_hanging(torch):
    """spin_limit = 1 makes contended locks give up: the call returns, no node stays locked."""
    import mvgpubtree_b200 as mv
    t = mv.gpu_blink_tree(pool_bytes=1 << 26, tile_width=8, spin_limit=1)
    keys = np.arange(1, 1 << 15, dtype=np.uint32)  # dense keys: heavy contention on few leaves
    t.insert(dev(torch, keys), dev(torch, keys))
    bits = t.check_errors(raise_on_error=False)
    assert bits & ~0x3 == 0  # only "pool" / "spin" bits may be set
    rep = t.validate_tree_structure(raise_on_error=False)
    assert rep["locked_nodes"] == 0
    # a writer that gave up after a split may leave its separator unposted: readers still reach
    # every key through the right links, so every find returns the stored value or a miss
    out = torch.empty(len(keys), dtype=torch.int32, device="cuda")
    t.find(dev(torch, keys), out)
    got = host(out)
    assert np.all((got == keys) | (got == SENT))


def test_cpp_drop_in_caller_runs(torch):
    """The C++ caller of include/gpu_btree.h (GpuBTree:: class names over the C ABI) gets the
    reference's known answers: finds and range counts at two snapshots."""
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    sys.path.insert(0, str(root / "tests" / "cpp"))
    exe = root / "tests" / "cpp" / "drop_in_example"
    if not exe.exists():
        from build import build
        build()
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and "OK" in out.stdout, out.stdout + out.stderr
