"""GPU tier: mixed op batches (persistent, graph-replayed and per-batch launches) vs the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need CUDA"
    return t


def dev(torch, a, dtype=None):
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        return torch.from_numpy(a.view(np.int64)).cuda()
    return torch.from_numpy(a.astype(np.uint32, copy=False).view(np.int32)).cuda()


def host(t):
    return t.cpu().numpy().view(np.uint32)


def _setup(torch, seed, n0, W=8, pool=2 << 30):
    import mvgpubtree_b200 as mv
    import oracle
    import workload as wl
    init = wl.distinct_keys(seed, 0, n0)
    vals = wl.values_for(init, 0)
    t = mv.gpu_versioned_btree(pool_bytes=pool, tile_width=W)
    t.insert(dev(torch, init), dev(torch, vals))
    m = oracle.MVMap(True)
    m.insert(init, vals)
    return t, m


def _run(torch, tree, plan, b, mode):
    ops = [dev(torch, b.type), dev(torch, b.key), dev(torch, b.arg), dev(torch, b.out_off),
           dev(torch, b.range_cap)]
    result = torch.zeros(b.num_ops, dtype=torch.int32, device="cuda")
    rout = torch.full((max(1, b.range_pairs) * 2,), -1, dtype=torch.int32, device="cuda")
    plan.run(b.batch_off, *ops, result, rout, mode=mode)
    tree.check_errors()
    return host(result), host(rout)


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("w", [8, 16])
def test_mixed_batches_match_oracle(torch, mode, w):
    import workload as wl
    seed, n0 = 31, 1 << 18
    t, m = _setup(torch, seed, n0, w)
    gen = wl.MixGenerator(seed, n0, stride=wl.stride_for(n0), batch_median=4096, batch_max=1 << 16)
    plan = t.batch_plan(1 << 22, 256)
    for rnd in range(2):  # the second round replays the captured graph / reuses the plan
        b = gen.generate(48)
        r, o = _run(torch, t, plan, b, mode)
        er, eo = m.run_batches(b)
        assert np.array_equal(r, er), f"round {rnd}: {np.count_nonzero(r != er)} results differ"
        assert np.array_equal(o, eo), f"round {rnd}: range output differs"
    rep = t.validate_tree_structure()
    assert rep["violations"] == 0 and rep["keys"] == m.size()


def test_batches_see_every_earlier_batch_and_snapshots_advance(torch):
    """Tiny batches exercise the batch-to-batch dependency of the persistent launch."""
    import mvgpubtree_b200 as mv
    import workload as wl
    seed, n0 = 5, 1 << 14
    t, m = _setup(torch, seed, n0)
    e0 = t.take_snapshot(); m.take_snapshot()
    gen = wl.MixGenerator(seed, n0, stride=wl.stride_for(n0), fixed_batch=64)
    b = gen.generate(200)
    plan = t.batch_plan(b.num_ops, 256)
    r, o = _run(torch, t, plan, b, mv.BATCH_PERSISTENT)
    er, eo = m.run_batches(b)
    assert np.array_equal(r, er) and np.array_equal(o, eo)
    assert t.take_snapshot() == m.take_snapshot() == e0 + 1 + 200


@pytest.mark.parametrize("dest", ["device", "pinned"])
def test_compact_range_output_packs_the_pairs_that_exist(torch, dest):
    """mvbt_batch_compact_ranges: every range query's first min(count, cap) pairs, in op order,
    packed contiguously (into device memory, or straight into pinned host memory)."""
    import workload as wl
    import mvgpubtree_b200 as mv
    initial, seed = 100_000, 29
    init = wl.distinct_keys(seed, 0, initial)
    t = mv.gpu_versioned_btree(pool_bytes=1 << 28)
    t.insert(torch.from_numpy(init.view(np.int32)).cuda(), torch.from_numpy(wl.values_for(init, 0).view(np.int32)).cuda())
    gen = wl.MixGenerator(seed, initial, stride=wl.stride_for(initial), batch_median=4096.0,
                          batch_min=256, batch_max=32768)
    b = gen.generate(12)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int64 if a.dtype == np.uint64 else np.int32)).cuda()
    ops = [d(b.type), d(b.key), d(b.arg), d(b.out_off), d(b.range_cap)]
    res = torch.empty(b.num_ops, dtype=torch.int32, device="cuda")
    rout = torch.full((b.range_pairs * 2,), -1, dtype=torch.int32, device="cuda")
    plan = t.batch_plan(b.num_ops, 12)
    plan.run(b.batch_off, *ops, res, rout)
    if dest == "device":
        comp = torch.full((b.range_pairs * 2,), -1, dtype=torch.int32, device="cuda")
        total = torch.zeros(1, dtype=torch.int64, device="cuda")
    else:
        comp = torch.full((b.range_pairs * 2,), -1, dtype=torch.int32).pin_memory()
        total = torch.zeros(1, dtype=torch.int64).pin_memory()
    plan.compact_ranges(b.num_ops, ops[0], res, ops[3], ops[4], rout, comp, total)
    torch.cuda.synchronize()
    r = res.cpu().numpy().view(np.uint32)
    ro = rout.cpu().numpy().view(np.uint32).reshape(-1, 2)
    rq = np.nonzero(b.type == 3)[0]
    want = np.concatenate([ro[int(b.out_off[i]): int(b.out_off[i]) + min(int(r[i]), int(b.range_cap[i]))]
                           for i in rq]) if rq.size else np.zeros((0, 2), np.uint32)
    got_total = int(total.cpu().numpy()[0])
    assert got_total == len(want) and got_total > 0
    got = comp.cpu().numpy().view(np.uint32).reshape(-1, 2)[:got_total]
    assert np.array_equal(got, want)


def test_compact_ranges_in_a_larger_plan_for_growing_op_counts(torch):
    """The packing scratch is sized for the plan's largest run on first use: packing a prefix of
    the ops and then all of them on a plan that holds more ops gives the right pairs both times."""
    import workload as wl
    import mvgpubtree_b200 as mv
    initial, seed = 100_000, 31
    init = wl.distinct_keys(seed, 0, initial)
    t = mv.gpu_versioned_btree(pool_bytes=1 << 28)
    t.insert(torch.from_numpy(init.view(np.int32)).cuda(), torch.from_numpy(wl.values_for(init, 0).view(np.int32)).cuda())
    gen = wl.MixGenerator(seed, initial, stride=wl.stride_for(initial), batch_median=4096.0,
                          batch_min=256, batch_max=32768)
    b = gen.generate(12)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int64 if a.dtype == np.uint64 else np.int32)).cuda()
    ops = [d(b.type), d(b.key), d(b.arg), d(b.out_off), d(b.range_cap)]
    res = torch.empty(b.num_ops, dtype=torch.int32, device="cuda")
    rout = torch.full((b.range_pairs * 2,), -1, dtype=torch.int32, device="cuda")
    plan = t.batch_plan(4 * b.num_ops, 12)
    plan.run(b.batch_off, *ops, res, rout)
    torch.cuda.synchronize()
    r = res.cpu().numpy().view(np.uint32)
    ro = rout.cpu().numpy().view(np.uint32).reshape(-1, 2)
    for n in (int(b.batch_off[6]), b.num_ops):
        comp = torch.full((b.range_pairs * 2,), -1, dtype=torch.int32, device="cuda")
        total = torch.zeros(1, dtype=torch.int64, device="cuda")
        plan.compact_ranges(n, ops[0], res, ops[3], ops[4], rout, comp, total)
        torch.cuda.synchronize()
        rq = np.nonzero(b.type[:n] == 3)[0]
        want = np.concatenate([ro[int(b.out_off[i]): int(b.out_off[i]) + min(int(r[i]), int(b.range_cap[i]))]
                               for i in rq]) if rq.size else np.zeros((0, 2), np.uint32)
        got_total = int(total.cpu().numpy()[0])
        assert got_total == len(want), n
        assert np.array_equal(comp.cpu().numpy().view(np.uint32).reshape(-1, 2)[:got_total], want), n
    assert t.check_errors() == 0


@pytest.mark.parametrize("w,bps", [(8, 0), (16, 6)])
def test_full_c4_step_at_4M_keys_matches_oracle_and_plain(torch, w, bps):
    """One step of the benchmark's batch law (256 batches, lognormal sizes median 16K ops, sigma
    1.5, clipped [1K, 4M]; erase 10 % / insert 20 % / find 50 % / range 20 %, L geometric mean 32)
    on a 4M-key tree: the persistent launch (at the benchmark's launch shapes) against the
    partitioned oracle, and against the plain per-batch launch on an identical tree -- every find
    value, range count and range-output word."""
    import mvgpubtree_b200 as mv
    import oracle
    import os
    import workload as wl
    seed, n0 = 20240611, 4_000_000
    init = wl.distinct_keys(seed, 0, n0)
    vals = wl.values_for(init, 0)
    gen = wl.MixGenerator(seed, n0, stride=wl.stride_for(40_000_000))
    b = gen.generate(256)
    assert b.num_ops > 5_000_000
    outs = []
    for mode in (mv.BATCH_PERSISTENT, mv.BATCH_PER_LAUNCH):
        t = mv.gpu_versioned_btree(pool_bytes=4 << 30, tile_width=w,
                                   blocks_per_sm=bps if mode == mv.BATCH_PERSISTENT else 0)
        t.insert(dev(torch, init), dev(torch, vals))
        plan = t.batch_plan(b.num_ops, 256)
        outs.append(_run(torch, t, plan, b, mode))
        rep = t.validate_tree_structure()
        assert rep["violations"] == 0
        plan.close()
        t.close()
    m = oracle.PartitionedMVMap(os.cpu_count() or 1, True)
    m.insert(init, vals)
    er, eo = m.run_batches(b)
    m.close()
    for name, (r, o) in zip(("persistent", "plain"), outs):
        assert np.array_equal(r, er), f"{name}: {np.count_nonzero(r != er)} of {r.size} results differ"
        assert np.array_equal(o, eo), f"{name}: {np.count_nonzero(o != eo)} range-output words differ"
    assert rep["keys"] == n0 + 1 + int(np.count_nonzero(b.type == 1)) - int(np.count_nonzero(b.type == 2))
