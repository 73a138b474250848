"""GPU tier: results identical to the reference implementation's own CUDA build on the same inputs.

oracle/_ref/ref_driver (built by oracle/ref_build.py from the reference's unmodified headers) runs
the reference through its public host API; this library runs the same workload through its C ABI;
checksums of every find result, range count and range pair are compared (oracle/refsums.py).
  * C1 shape: plain B-link tree, insert then finds (half present, half never inserted).
  * C2 shape: versioned tree, finds of the same queries at a snapshot before and after updates.
  * C3 shape: versioned tree, range queries at a snapshot before and after new inserts (a
    deterministic sequence; the reference's concurrent_insert_range is not run).
  * C4 shape: versioned tree, mixed batches with one snapshot per batch. The reference issues each
    batch in its plain form (take_snapshot, find(ts), range_query(ts), insert, erase); this library
    runs all batches in one persistent launch. A final snapshot reads the whole key space.
"""
import numpy as np
import pytest

from oracle.refsums import DRIVER, find_sum, count_sum, pairs_sum, run_driver, step_sums

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not DRIVER.exists(), reason="reference build not present (oracle/ref_build.py)")]


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need CUDA"
    return t


def dev(torch, a):
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        return torch.from_numpy(a.view(np.int64)).cuda()
    return torch.from_numpy(a.astype(np.uint32).view(np.int32)).cuda()


def host(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("w", [8, 16])
def test_plain_tree_finds_match_reference_build(torch, w):
    import workload as wl
    import mvgpubtree_b200 as mv
    n, seed = 1 << 16, 7
    ref = run_driver("c1", "--n", str(n), "--seed", str(seed))
    keys = wl.distinct_keys(seed, 0, n)
    vals = wl.values_for(keys, seed)
    hits = wl.shuffle(seed + 1, keys)[: n // 2]
    miss = wl.distinct_keys(seed, wl.MISS_INDEX_BASE, n - n // 2)
    q = wl.shuffle(seed + 2, np.concatenate([hits, miss]))
    t = mv.gpu_blink_tree(pool_bytes=1 << 28, tile_width=w)
    t.insert(dev(torch, keys), dev(torch, vals))
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    t.find(dev(torch, q), out)
    assert t.check_errors() == 0
    assert find_sum(np.arange(n), host(out)) == ref["find_checksum"]


@pytest.mark.parametrize("w", [8, 16])
def test_mixed_batches_match_reference_build(torch, w):
    import workload as wl
    import mvgpubtree_b200 as mv
    initial, seed, nb, warm, steps, chunks = 200_000, 5, 24, 1, 1, 64
    stride = wl.stride_for(initial)
    gen_args = dict(batch_median=2048.0, batch_min=64, batch_max=16384)
    ref = run_driver("c4", "--initial", str(initial), "--batches", str(nb), "--steps", str(steps),
                     "--warmup", str(warm), "--seed", str(seed), "--stride", str(stride),
                     "--median", "2048", "--batch-min", "64", "--batch-max", "16384",
                     "--final-chunks", str(chunks))
    init = wl.distinct_keys(seed, 0, initial)
    vals = wl.values_for(init, 0)
    gen = wl.MixGenerator(seed, initial, stride=stride, **gen_args)
    t = mv.gpu_versioned_btree(pool_bytes=1 << 30, tile_width=w)
    t.insert(dev(torch, init), dev(torch, vals))
    sums = []
    plan = None
    for _ in range(warm + steps):
        b = gen.generate(nb)
        if plan is None:
            plan = t.batch_plan(4 * b.num_ops + 65536, nb)
        res = torch.empty(b.num_ops, dtype=torch.int32, device="cuda")
        rout = torch.full((max(1, b.range_pairs) * 2,), -1, dtype=torch.int32, device="cuda")
        plan.run(b.batch_off, dev(torch, b.type), dev(torch, b.key), dev(torch, b.arg),
                 dev(torch, b.out_off), dev(torch, b.range_cap), res, rout, mode=mv.BATCH_PERSISTENT)
        assert t.check_errors() == 0
        sums.append(step_sums(b, host(res), host(rout).reshape(-1, 2)))
    assert sums == ref["step_checksums"]
    # final state: the whole key space at a final snapshot, in the driver's chunks and slot size
    live = gen.present
    span = (0xFFFFFFFF - 1 + chunks - 1) // chunks
    slot = min((live // chunks) * 2 + 1024, 1 << 24)
    lo = np.array([1 + c * span for c in range(chunks)], np.uint64)
    hi = np.minimum(lo + span, 0xFFFFFFFF)
    S = t.take_snapshot()
    pairs = torch.full((chunks * slot * 2,), -1, dtype=torch.int32, device="cuda")
    counts = torch.empty(chunks, dtype=torch.int32, device="cuda")
    t.range_query(dev(torch, lo.astype(np.uint32)), dev(torch, hi.astype(np.uint32)), pairs, counts,
                  slot, chunks, S)
    cnt = host(counts)
    idx = np.arange(chunks)
    final = [count_sum(idx, cnt),
             pairs_sum(idx, np.minimum(cnt, slot), idx * slot, host(pairs).reshape(-1, 2))]
    assert final == ref["final"]
    assert int(cnt.sum()) == live


@pytest.mark.parametrize("w", [8, 16])
def test_versioned_finds_at_two_snapshots_match_reference_build(torch, w):
    """C2 shape: insert, snapshot S0, in-place updates of an eighth of the keys, snapshot S1,
    the same hit/miss queries at S0 and at S1."""
    import workload as wl
    import mvgpubtree_b200 as mv
    n, seed = 1 << 17, 13
    u = n // 8
    ref = run_driver("c2", "--initial", str(n), "--updates", str(u), "--seed", str(seed))
    keys = wl.distinct_keys(seed, 0, n)
    upd = wl.shuffle(seed + 3, keys)[:u]
    hits = wl.shuffle(seed + 1, keys)[: n // 2]
    miss = wl.distinct_keys(seed, wl.MISS_INDEX_BASE, n - n // 2)
    q = wl.shuffle(seed + 2, np.concatenate([hits, miss]))
    t = mv.gpu_versioned_btree(pool_bytes=1 << 28, tile_width=w)
    t.insert(dev(torch, keys), dev(torch, wl.values_for(keys, seed)))
    s0 = t.take_snapshot()
    t.insert(dev(torch, upd), dev(torch, wl.values_for(upd, seed ^ 1)))
    s1 = t.take_snapshot()
    sums = []
    for s in (s0, s1):
        out = torch.empty(n, dtype=torch.int32, device="cuda")
        t.find(dev(torch, q), out, timestamp=s)
        sums.append(find_sum(np.arange(n), host(out)))
    assert t.check_errors() == 0
    assert sums == ref["find_checksums"]


def c3_case(seed, n, ops, u, L):
    import workload as wl
    stride = wl.stride_for(n)
    n_ins = int(ops * u)
    n_rq = ops - n_ins
    keys = wl.distinct_keys(seed, 0, n)
    ins = wl.distinct_keys(seed, n, n_ins)
    lo = wl.uniform_keys(seed + 1, n_rq)
    return dict(stride=stride, n_ins=n_ins, n_rq=n_rq, keys=keys, vals=wl.values_for(keys, seed), ins=ins,
                ivals=wl.values_for(ins, seed), lo=lo, hi=wl.upper_bounds(lo, L, stride))


def range_sums(cnt, pairs, slot):
    idx = np.arange(cnt.size)
    return [count_sum(idx, cnt), pairs_sum(idx, np.minimum(cnt, slot), idx * slot, pairs.reshape(-1, 2))]


@pytest.mark.parametrize("w", [8, 16])
@pytest.mark.parametrize("u,L", [(0.5, 8), (0.9, 128)])
def test_insert_then_ranges_match_reference_build(torch, w, u, L, tmp_path):
    """C3 shape: insert, snapshot S0, new keys inserted, snapshot S1, the same range queries at S0
    and at S1 (4L + 64 pairs per query, more than any of these queries returns). The reference's
    concurrent_insert_range lets each query tile take its own snapshot, so its results depend on
    timing (and it is not run: it raised an illegal memory access on a B200 with in-bounds
    inputs); the check is this deterministic sequence.

    This library and the oracle agree on every query. The reference agrees with both when its
    second insert is in place (its ViB form). With the out-of-place form (VoB) its range counts
    at S0 include some keys inserted after S0 (1-3 extra in ~0.02-3 % of queries here); at S1 it
    agrees. That case is recorded as an expected failure of the reference, not of this library."""
    import mvgpubtree_b200 as mv
    import oracle
    n, seed, ops = 1 << 18, 29, 60_000
    c = c3_case(seed, n, ops, u, L)
    ref = run_driver("c3", "--initial", str(n), "--seed", str(seed), "--stride", str(c["stride"]),
                     "--combos", f"{c['n_ins']}:{c['n_rq']}:{L}:{2 * L}",
                     "--dump", str(tmp_path / "ref"))["runs"][0]
    slot = 4 * L + 64
    assert ref["check_slot"] == slot and ref["max_count"] <= slot
    t = mv.gpu_versioned_btree(pool_bytes=1 << 28, tile_width=w)
    t.insert(dev(torch, c["keys"]), dev(torch, c["vals"]))
    s0 = t.take_snapshot()
    t.insert(dev(torch, c["ins"]), dev(torch, c["ivals"]))
    s1 = t.take_snapshot()
    ours = []
    for s in (s0, s1):
        pairs = torch.full((c["n_rq"] * slot * 2,), -1, dtype=torch.int32, device="cuda")
        counts = torch.empty(c["n_rq"], dtype=torch.int32, device="cuda")
        t.range_query(dev(torch, c["lo"]), dev(torch, c["hi"]), pairs, counts, slot, c["n_rq"], s)
        ours += range_sums(host(counts), host(pairs), slot)
    assert t.check_errors() == 0
    m = oracle.MVMap(True)
    m.insert(c["keys"], c["vals"])
    o0 = m.take_snapshot()
    m.insert(c["ins"], c["ivals"])
    o1 = m.take_snapshot()
    expect, oc = [], []
    for s in (o0, o1):
        pairs, counts = m.range_query(c["lo"], c["hi"], slot, s)
        expect += range_sums(counts, pairs, slot)
        oc.append(counts)
    assert ours == expect
    assert ref["checksums"] == ours  # reference, second insert in place
    vob = ref["checksums_out_of_place"]
    assert vob[2:] == ours[2:]  # reference, out of place: at S1
    if vob[:2] != ours[:2]:
        rc = np.fromfile(tmp_path / "ref_vob_s0.u32", np.uint32)
        bad = np.nonzero(rc != oc[0])[0]
        extra = rc[bad].astype(np.int64) - oc[0][bad].astype(np.int64)
        newer = oc[1][bad].astype(np.int64) - oc[0][bad].astype(np.int64)
        assert np.all(extra > 0) and np.all(extra <= newer), "the reference's extra keys are not later inserts"
        pytest.xfail(f"reference out-of-place insert: {bad.size} of {c['n_rq']} range counts at the earlier "
                     f"snapshot include {int(extra.min())}-{int(extra.max())} keys inserted after it")
