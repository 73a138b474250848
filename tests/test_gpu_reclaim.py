"""GPU tier: reclamation of version copies (mvbt_reclaim).

* Mixed batches with a reclaim pass after every step give the same results, bit for bit, as the
  same batches on a tree that keeps every version, while the allocation high-water mark stops
  growing (freed copies are handed out again).
* A reclaim with watermark S keeps snapshot S readable (checked against the oracle); a later
  reclaim of everything keeps the newest state.
* Without config.reclaim the call is refused.
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
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        return torch.from_numpy(a.view(np.int64)).cuda()
    return torch.from_numpy(a.astype(np.uint32).view(np.int32)).cuda()


def host(t):
    return t.cpu().numpy().view(np.uint32)


def test_reclaim_needs_the_config_flag(torch):
    import mvgpubtree_b200 as mv
    t = mv.gpu_versioned_btree(pool_bytes=1 << 26)
    with pytest.raises(mv.MVBTError):
        t.reclaim()
    p = mv.gpu_blink_tree(pool_bytes=1 << 26, reclaim=True)
    p.reclaim()  # the plain tree makes no copies: a no-op
    assert p.stats()["reclaimed"] == 0


@pytest.mark.parametrize("w", [8, 16])
def test_batches_with_reclaim_match_and_memory_stays_flat(torch, w):
    import workload as wl
    import mvgpubtree_b200 as mv
    initial, seed, nb, steps = 400_000, 9, 32, 8
    init = wl.distinct_keys(seed, 0, initial)
    vals = wl.values_for(init, 0)
    gen = wl.MixGenerator(seed, initial, stride=wl.stride_for(initial), batch_median=4096.0,
                          batch_min=256, batch_max=32768)
    batches = [gen.generate(nb) for _ in range(steps)]
    trees = {"reclaim": mv.gpu_versioned_btree(pool_bytes=1 << 30, tile_width=w, reclaim=True),
             "keep": mv.gpu_versioned_btree(pool_bytes=1 << 30, tile_width=w)}
    max_ops = max(b.num_ops for b in batches)
    plans = {}
    for k, t in trees.items():
        t.insert(dev(torch, init), dev(torch, vals))
        plans[k] = t.batch_plan(max_ops, nb)
    used = {k: [] for k in trees}
    for s, b in enumerate(batches):
        out = {}
        ops = [dev(torch, a) for a in (b.type, b.key, b.arg, b.out_off, b.range_cap)]
        for k, t in trees.items():
            res = torch.empty(b.num_ops, dtype=torch.int32, device="cuda")
            rout = torch.full((max(1, b.range_pairs) * 2,), -1, dtype=torch.int32, device="cuda")
            plans[k].run(b.batch_off, *ops, res, rout, mode=mv.BATCH_PERSISTENT)
            if k == "reclaim":
                t.reclaim()  # every snapshot of this step is finished
            assert t.check_errors() == 0
            out[k] = (host(res), host(rout))
            used[k].append(t.compute_memory_usage()["nodes_allocated"])
        assert np.array_equal(out["reclaim"][0], out["keep"][0]), f"step {s} results"
        assert np.array_equal(out["reclaim"][1], out["keep"][1]), f"step {s} range output"
    st = trees["reclaim"].stats()
    assert st["reclaimed"] > 0 and st["reused"] > 0 and st["log_dropped"] == 0
    grow_r = used["reclaim"][-1] - used["reclaim"][2]
    grow_k = used["keep"][-1] - used["keep"][2]
    assert grow_r < 0.2 * grow_k, (used, st)
    # the newest state agrees key for key, and the reclaimed tree is well formed
    q = np.concatenate([init, wl.distinct_keys(seed, wl.MISS_INDEX_BASE, 1000)])
    outs = []
    for t in trees.values():
        o = torch.empty(len(q), dtype=torch.int32, device="cuda")
        t.find(dev(torch, q), o)
        outs.append(host(o))
    assert np.array_equal(outs[0], outs[1])
    rep = trees["reclaim"].validate_tree_structure()
    assert rep["violations"] == 0 and rep["locked_nodes"] == 0


@pytest.mark.parametrize("w", [8, 16])
def test_reclaim_watermark_keeps_that_snapshot(torch, w):
    import workload as wl
    import mvgpubtree_b200 as mv
    import oracle
    seed, n0 = 13, 1 << 16
    keys = wl.distinct_keys(seed, 0, n0)
    t = mv.gpu_versioned_btree(pool_bytes=1 << 28, tile_width=w, reclaim=True)
    m = oracle.MVMap(True)
    t.insert(dev(torch, keys), dev(torch, wl.values_for(keys, seed)))
    m.insert(keys, wl.values_for(keys, seed))
    held = None
    for r in range(5):
        s = t.take_snapshot()
        assert s == m.take_snapshot()
        if r == 2:
            held = s
        upd = wl.shuffle(seed + r, keys)[: n0 // 3]
        t.insert(dev(torch, upd), dev(torch, wl.values_for(upd, seed + 10 + r)))
        m.insert(upd, wl.values_for(upd, seed + 10 + r))
        er = wl.shuffle(seed + 20 + r, keys)[: n0 // 20]
        t.erase(dev(torch, er))
        m.erase(er)
    t.reclaim(held)  # copies read only below the held snapshot go
    assert t.check_errors() == 0
    assert t.stats()["reclaimed"] > 0
    for ts in (held, mv.LATEST):
        out = torch.empty(n0, dtype=torch.int32, device="cuda")
        t.find(dev(torch, keys), out, timestamp=ts)
        assert np.array_equal(host(out), m.find(keys, ts)), f"snapshot {ts}"
    t.reclaim()
    out = torch.empty(n0, dtype=torch.int32, device="cuda")
    t.find(dev(torch, keys), out)
    assert np.array_equal(host(out), m.find(keys, mv.LATEST))
    assert t.validate_tree_structure()["violations"] == 0


@pytest.mark.parametrize("mode", [0, 2])
@pytest.mark.parametrize("w", [8, 16])
def test_reclamation_inside_persistent_runs(torch, w, mode):
    """mvbt_batch_plan_set_reclaim: copies are freed while the persistent launch runs (by warps
    without work, once every snapshot that reads them is finished) and handed out again. Results
    are bit-identical to a tree that keeps every version, no pass between launches is needed, the
    node count stops growing, and the memory series of each run is consistent."""
    import workload as wl
    import mvgpubtree_b200 as mv
    initial, seed, nb, steps = 400_000, 19, 48, 8
    init = wl.distinct_keys(seed, 0, initial)
    vals = wl.values_for(init, 0)
    gen = wl.MixGenerator(seed, initial, stride=wl.stride_for(initial), batch_median=4096.0,
                          batch_min=256, batch_max=32768)
    batches = [gen.generate(nb) for _ in range(steps)]
    trees = {"inside": mv.gpu_versioned_btree(pool_bytes=1 << 30, tile_width=w, reclaim=True),
             "keep": mv.gpu_versioned_btree(pool_bytes=1 << 30, tile_width=w)}
    max_ops = max(b.num_ops for b in batches)
    plans = {}
    for k, t in trees.items():
        t.insert(dev(torch, init), dev(torch, vals))
        plans[k] = t.batch_plan(max_ops, nb)
    plans["inside"].set_reclaim(True)
    used = {k: [] for k in trees}
    for s, b in enumerate(batches):
        out = {}
        ops = [dev(torch, a) for a in (b.type, b.key, b.arg, b.out_off, b.range_cap)]
        for k, t in trees.items():
            res = torch.empty(b.num_ops, dtype=torch.int32, device="cuda")
            rout = torch.full((max(1, b.range_pairs) * 2,), -1, dtype=torch.int32, device="cuda")
            plans[k].run(b.batch_off, *ops, res, rout, mode=mode)
            assert t.check_errors() == 0
            out[k] = (host(res), host(rout))
            used[k].append(t.compute_memory_usage()["nodes_allocated"])
        assert np.array_equal(out["inside"][0], out["keep"][0]), f"step {s} results"
        assert np.array_equal(out["inside"][1], out["keep"][1]), f"step {s} range output"
        ser = plans["inside"].memory_series()
        assert ser.shape == (nb, 4)
        assert np.all(np.diff(ser[:, 0].astype(np.int64)) == 1)          # one epoch per batch
        assert np.all(np.diff(ser[:, 3].astype(np.int64)) >= 0)          # freed so far: monotone
        assert np.all(ser[:, 1] >= ser[:, 2])                            # live nodes >= 0
    st = trees["inside"].stats()
    assert st["reclaimed"] > 0 and st["reused"] > 0 and st["log_dropped"] == 0, st
    grow_i = used["inside"][-1] - used["inside"][2]
    grow_k = used["keep"][-1] - used["keep"][2]
    assert grow_i < 0.2 * grow_k, (used, st)
    q = np.concatenate([init, wl.distinct_keys(seed, wl.MISS_INDEX_BASE, 1000)])
    outs = []
    for t in trees.values():
        o = torch.empty(len(q), dtype=torch.int32, device="cuda")
        t.find(dev(torch, q), o)
        outs.append(host(o))
    assert np.array_equal(outs[0], outs[1])
    rep = trees["inside"].validate_tree_structure()
    assert rep["violations"] == 0 and rep["locked_nodes"] == 0


def test_reclamation_inside_runs_keeps_a_held_snapshot(torch):
    """With a snapshot held outside the runs (the watermark), the copies it reads survive the
    runs' reclamation: finds at it match the oracle after several steps."""
    import workload as wl
    import mvgpubtree_b200 as mv
    import oracle
    initial, seed, nb = 200_000, 23, 24
    init = wl.distinct_keys(seed, 0, initial)
    vals = wl.values_for(init, 0)
    t = mv.gpu_versioned_btree(pool_bytes=1 << 29, reclaim=True)
    t.insert(dev(torch, init), dev(torch, vals))
    m = oracle.MVMap(True)
    m.insert(init, vals)
    gen = wl.MixGenerator(seed, initial, stride=wl.stride_for(initial), batch_median=2048.0,
                          batch_min=256, batch_max=8192)
    plan = t.batch_plan(1 << 20, nb)
    held = None
    for s in range(6):
        if s == 2:
            held = t.take_snapshot(); assert held == m.take_snapshot()
        plan.set_reclaim(True, 0xFFFFFFFF if held is None else held)
        b = gen.generate(nb)
        ops = [dev(torch, a) for a in (b.type, b.key, b.arg, b.out_off, b.range_cap)]
        res = torch.empty(b.num_ops, dtype=torch.int32, device="cuda")
        rout = torch.full((max(1, b.range_pairs) * 2,), -1, dtype=torch.int32, device="cuda")
        plan.run(b.batch_off, *ops, res, rout, mode=mv.BATCH_PERSISTENT)
        er, eo = m.run_batches(b)
        assert np.array_equal(host(res), er) and np.array_equal(host(rout), eo), s
        assert t.check_errors() == 0
    assert t.stats()["reclaimed"] > 0
    out = torch.empty(initial, dtype=torch.int32, device="cuda")
    t.find(dev(torch, init), out, timestamp=held)
    assert np.array_equal(host(out), m.find(init, held))
