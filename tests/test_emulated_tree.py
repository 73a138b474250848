"""CPU tier: the device tree code (include/mvbt_device.cuh) compiled for the host and run with
W host threads per tile and several concurrent tiles (tests/emu), checked against the oracle.

This exercises the lock, split, copy-on-write and snapshot-read protocols on the CPU; the GPU
tier repeats the same checks on the B200.
"""
import numpy as np
import pytest

from cases import EmuDriver, load_cases, replay


def _case_params():
    _, index = load_cases()
    out = []
    for c in index:
        for kind in c["kinds"]:
            out.append(pytest.param(c["name"], kind, 8, id=f"{c['name']}-{kind}-w8"))
    # W=16 on a representative subset to keep the CPU tier short
    for name, kind in (("btree_EraseAllInsertAllTest", "versioned"), ("versioning_RangeQueryTest", "versioned"),
                       ("find_blink_test", "blink")):
        out.append(pytest.param(name, kind, 16, id=f"{name}-{kind}-w16"))
    return out


@pytest.mark.parametrize("name,kind,w", _case_params())
def test_emulated_tree_matches_reference_known_answers(name, kind, w):
    z, index = load_cases()
    case = next(c for c in index if c["name"] == name)
    replay(EmuDriver(kind == "versioned", tile_width=w, tiles=8), z, case)


@pytest.mark.parametrize("w", [8, 16])
def test_emulated_concurrent_insert_range_at_launch_snapshot(w):
    from emu import EmuTree
    import workload as wl
    import oracle
    seed, n0, L = 3, 3000, 8
    keys = wl.distinct_keys(seed, 0, n0)
    vals = wl.values_for(keys, seed)
    t = EmuTree(True, capacity=1 << 15, tiles=8, W=w)
    m = oracle.MVMap(True)
    t.insert(keys, vals)
    m.insert(keys, vals)
    ins = wl.distinct_keys(seed, n0, 1500)
    lo = wl.uniform_keys(seed, 600)
    hi = wl.upper_bounds(lo, L, wl.stride_for(n0))
    pairs, counts = t.insert_range(ins, wl.values_for(ins, seed), lo, hi, 32)
    assert t.errors == 0
    s = m.take_snapshot()
    ep, ec = m.range_query(lo, hi, 32, s)
    assert np.array_equal(counts, ec)
    mask = np.arange(32)[None, :] < np.minimum(ec, 32)[:, None]
    assert np.array_equal(pairs[mask], ep[mask])
    m.insert(ins, wl.values_for(ins, seed))
    q = np.concatenate([keys, ins])
    assert np.array_equal(t.find(q), m.find(q))
    rep = t.validate()
    assert rep["violations"] == 0 and rep["locked_nodes"] == 0 and rep["keys"] == n0 + 1500 + 1
    rep0 = t.validate(s)
    assert rep0["violations"] == 0 and rep0["keys"] == n0 + 1


@pytest.mark.parametrize("w", [8, 16])
def test_emulated_find_erase_newest_state(w):
    """Finds of the newest state running beside erases that shift leaf pairs (the plain tree's
    concurrent_find_erase): a find returns the key's value, or not-found only for an erased key
    (include/validation.hpp:106-149 of the reference accepts exactly these)."""
    from emu import EmuTree
    import workload as wl
    import oracle
    seed, n0 = 21, 6000
    keys = wl.distinct_keys(seed, 0, n0)
    vals = wl.values_for(keys, seed)
    t = EmuTree(False, capacity=1 << 15, tiles=8, W=w)
    t.insert(keys, vals)
    er = wl.shuffle(seed + 1, keys)[: n0 // 2]
    fk = wl.shuffle(seed + 2, keys)
    got = t.find_erase(fk, er)
    assert t.errors == 0
    expect = wl.values_for(fk, seed)
    erased = np.isin(fk, er)
    assert np.all((got == expect) | (erased & (got == 0xFFFFFFFF)))
    m = oracle.MVMap(False)
    m.insert(keys, vals)
    m.erase(er)
    assert np.array_equal(t.find(keys), m.find(keys))


@pytest.mark.parametrize("w", [8, 16])
def test_emulated_reclaim_keeps_live_snapshots_and_reuses_nodes(w):
    """Rounds of snapshot s, updates and erases, then a reclaim with watermark s: finds at s and
    at the newest state still match the oracle, freed copies are handed out again, and the
    allocation high-water mark stops growing."""
    from emu import EmuTree
    import workload as wl
    import oracle
    seed, n0 = 31, 3000
    keys = wl.distinct_keys(seed, 0, n0)
    t = EmuTree(True, capacity=1 << 14, tiles=8, W=w, reclaim=True)
    m = oracle.MVMap(True)
    t.insert(keys, wl.values_for(keys, seed))
    m.insert(keys, wl.values_for(keys, seed))
    bumps, copies = [], []
    for r in range(6):
        s = t.snapshot()
        assert s == m.take_snapshot()
        upd = wl.shuffle(seed + r, keys)[:1000]
        t.insert(upd, wl.values_for(upd, seed + 100 + r))
        m.insert(upd, wl.values_for(upd, seed + 100 + r))
        er = wl.shuffle(seed + 50 + r, keys)[:200]
        t.erase(er)
        m.erase(er)
        t.reclaim(s)  # copies made before s are unreadable now; s itself stays readable
        assert t.errors == 0
        assert np.array_equal(t.find(keys, s), m.find(keys, s)), f"round {r} at snapshot {s}"
        assert np.array_equal(t.find(keys), m.find(keys)), f"round {r} newest state"
        bumps.append(t.bump)
        copies.append(t.stats()["cow"])
    st = t.stats()
    assert st["reclaimed"] > 0 and st["reused"] > 0 and st["log_dropped"] == 0
    # the last three rounds made many copies but allocated few new nodes: freed ones were reused
    assert bumps[-1] - bumps[2] < 0.25 * (copies[-1] - copies[2])
    t.reclaim()  # everything older than the newest state
    assert np.array_equal(t.find(keys), m.find(keys))
    rep = t.validate()
    assert rep["violations"] == 0 and rep["locked_nodes"] == 0


def test_emulated_updates_erases_keep_old_snapshots():
    from emu import EmuTree
    import workload as wl
    import oracle
    seed, n0 = 9, 4000
    keys = wl.distinct_keys(seed, 0, n0)
    t = EmuTree(True, capacity=1 << 15, tiles=8, W=8)
    m = oracle.MVMap(True)
    t.insert(keys, wl.values_for(keys, seed)); m.insert(keys, wl.values_for(keys, seed))
    snaps = []
    for r in range(3):
        snaps.append(t.snapshot()); m.take_snapshot()
        upd = wl.shuffle(seed + r, keys)[:800]
        t.insert(upd, wl.values_for(upd, seed + 100 + r)); m.insert(upd, wl.values_for(upd, seed + 100 + r))
        er = wl.shuffle(seed + 50 + r, keys)[:300]
        t.erase(er); m.erase(er)
        more = wl.distinct_keys(seed, n0 + 1000 * r, 500)
        t.insert(more, wl.values_for(more, seed)); m.insert(more, wl.values_for(more, seed))
    assert t.errors == 0
    q = np.concatenate([keys, wl.distinct_keys(seed, n0, 3000)])
    for s in snaps + [0xFFFFFFFF]:
        assert np.array_equal(t.find(q, s), m.find(q, s)), f"snapshot {s}"
        assert t.validate(s)["violations"] == 0


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("w", [8, 16])
def test_emulated_mixed_batches_match_oracle(mode, w):
    """Mixed erase/insert/find/range batches, one snapshot per batch (persistent worker loop
    with the writes-of-previous-batch dependency, and the per-batch mode)."""
    from emu import EmuTree
    import workload as wl
    import oracle
    seed, n0 = 12, 4000
    gen = wl.MixGenerator(seed, n0, stride=wl.stride_for(n0), batch_median=250, batch_min=1,
                          batch_max=2500, batch_sigma=1.2)
    b = gen.generate(12)
    init = wl.distinct_keys(seed, 0, n0)
    t = EmuTree(True, capacity=1 << 15, tiles=8, W=w)
    m = oracle.MVMap(True)
    t.insert(init, wl.values_for(init, 0))
    m.insert(init, wl.values_for(init, 0))
    r, o = t.run_batches(b, mode)
    er, eo = m.run_batches(b)
    assert t.errors == 0
    assert np.array_equal(r, er) and np.array_equal(o, eo)
    assert t.validate()["violations"] == 0


@pytest.mark.parametrize("w", [8, 16])
def test_emulated_sorted_runs_match_oracle(w):
    """The sorted batch front-end's device code (per-tile runs of sorted keys, each op starting
    from the deepest covering node of the previous op's path): inserts into a growing tree with
    repeated keys (the last occurrence wins), updates after a snapshot, erases, and finds and
    range queries at both snapshots, against the oracle."""
    from emu import EmuTree
    import workload as wl
    import oracle
    seed, n0 = 11, 4000
    keys = wl.distinct_keys(seed, 0, n0)
    vals = wl.values_for(keys, seed)
    rng = np.random.default_rng(seed)
    dup = rng.choice(n0, 300, replace=False)
    ins_k = np.concatenate([keys, keys[dup]])          # 300 keys appear twice
    ins_v = np.concatenate([vals, wl.values_for(keys[dup], seed ^ 7)])
    t = EmuTree(True, capacity=1 << 15, tiles=6, W=w)
    m = oracle.MVMap(True)
    t.sorted_run("insert", ins_k, ins_v)
    m.insert(ins_k, ins_v)  # in order: the second occurrence wins
    s0 = t.snapshot(); assert s0 == m.take_snapshot()
    upd = keys[rng.choice(n0, 900, replace=False)]
    t.sorted_run("insert", upd, wl.values_for(upd, seed ^ 1))
    m.insert(upd, wl.values_for(upd, seed ^ 1))
    er = keys[rng.choice(n0, 700, replace=False)]
    t.sorted_run("erase", er)
    m.erase(er)
    assert t.errors == 0
    s1 = t.snapshot(); assert s1 == m.take_snapshot()
    q = np.concatenate([keys, wl.distinct_keys(seed, wl.MISS_INDEX_BASE, 500)])
    q = wl.shuffle(seed, q)
    lo = wl.uniform_keys(seed + 5, 800)
    hi = wl.upper_bounds(lo, 16, wl.stride_for(n0))
    for ts in (s0, s1):
        assert np.array_equal(t.sorted_run("find", q, ts=ts), m.find(q, ts)), ts
        assert np.array_equal(t.sorted_run("qfind", q, ts=ts), m.find(q, ts)), ts
        assert np.array_equal(t.find(q, ts, quiescent=True), m.find(q, ts)), ts
        ep, ec = m.range_query(lo, hi, 48, ts)
        mask = np.arange(48)[None, :] < np.minimum(ec, 48)[:, None]
        for kind in ("range", "qrange"):
            pairs, counts = t.sorted_run(kind, lo, hi, avg_len=48, ts=ts)
            assert np.array_equal(counts, ec), (kind, ts)
            assert np.array_equal(pairs[mask], ep[mask]), (kind, ts)
        pairs, counts = t.range(lo, hi, 48, ts, quiescent=True)
        assert np.array_equal(counts, ec), ts
        assert np.array_equal(pairs[mask], ep[mask]), ts
    rep = t.validate()
    assert rep["violations"] == 0 and rep["locked_nodes"] == 0 and rep["keys"] == m.size()


@pytest.mark.parametrize("w", [8, 16])
def test_emulated_reclamation_inside_persistent_runs(w):
    """Reclamation inside the persistent batched run: idle warps free the copies that no snapshot
    reads any more, and the run's own writes allocate them again. Results stay identical to the
    oracle's, the node high-water mark stays well below a run without reclamation, and the memory
    samples count freed nodes. Then a snapshot held outside the runs (the watermark) stays exact
    while later runs go on."""
    from emu import EmuTree
    import workload as wl
    import oracle
    seed, n0 = 17, 3000
    init = wl.distinct_keys(seed, 0, n0)
    vals = wl.values_for(init, 0)
    trees = {}
    for rc in (False, True):
        trees[rc] = EmuTree(True, capacity=1 << 15, tiles=8, W=w, reclaim=True)
        trees[rc].insert(init, vals)
    m = oracle.MVMap(True)
    m.insert(init, vals)
    gen = wl.MixGenerator(seed, n0, stride=wl.stride_for(n0), fixed_batch=96)
    held = None
    for rnd in range(8):
        if rnd == 5:  # from here on the caller reads this snapshot outside the runs
            held = trees[True].snapshot(); trees[False].snapshot(); m.take_snapshot()
        b = gen.generate(24)
        er, eo = m.run_batches(b)
        series = np.zeros((24, 4), np.uint64)
        for rc, t in trees.items():
            r, o = t.run_batches(b, reclaim=rc, watermark=0xFFFFFFFF if held is None else held,
                                 series=series if rc else None)
            assert t.errors == 0
            assert np.array_equal(r, er), (rnd, rc, np.count_nonzero(r != er))
            assert np.array_equal(o, eo), (rnd, rc)
        assert np.all(series[:, 0] == np.arange(24) + series[0, 0])  # epochs of the batches' writes
        assert np.all(np.diff(series[:, 3].astype(np.int64)) >= 0)  # nodes freed so far: monotone
        if rnd == 4:
            st = trees[True].stats()
            assert st["reclaimed"] > 0 and st["reused"] > 0, st
            assert trees[True].bump < trees[False].bump, (trees[True].bump, trees[False].bump)
    q = np.concatenate([init, wl.distinct_keys(seed, wl.MISS_INDEX_BASE, 300)])
    assert np.array_equal(trees[True].find(q, held), m.find(q, held))
    for t in trees.values():
        rep = t.validate()
        assert rep["violations"] == 0 and rep["locked_nodes"] == 0 and rep["keys"] == m.size()
