"""GPU tier: copies of a tree (mvbt_clone, mvbt_save / mvbt_load), launch shapes of the batch path
and the autotuner that picks one.

* A clone reads exactly like its source at every snapshot and is independent afterwards.
* A saved and loaded tree reads like the original at every snapshot and continues identically.
* Every launch shape (tile width 8 / 16, full occupancy or register-capped) gives bit-identical
  batch results.
* Autotuning runs on clones and leaves the tree as it was.
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


def find(torch, t, keys, ts):
    out = torch.empty(len(keys), dtype=torch.int32, device="cuda")
    t.find(dev(torch, keys), out, timestamp=ts)
    return host(out)


def build(torch, mv, wl, seed=41, n0=1 << 16, reclaim=True):
    keys = wl.distinct_keys(seed, 0, n0)
    t = mv.gpu_versioned_btree(pool_bytes=1 << 28, reclaim=reclaim)
    t.insert(dev(torch, keys), dev(torch, wl.values_for(keys, seed)))
    s0 = t.take_snapshot()
    upd = wl.shuffle(seed + 1, keys)[: n0 // 4]
    t.insert(dev(torch, upd), dev(torch, wl.values_for(upd, seed + 1)))
    t.erase(dev(torch, wl.shuffle(seed + 2, keys)[: n0 // 8]))
    s1 = t.take_snapshot()
    return t, keys, (s0, s1)


def test_clone_reads_like_the_source_and_is_independent(torch):
    import workload as wl
    import mvgpubtree_b200 as mv
    t, keys, snaps = build(torch, mv, wl)
    c = t.clone()
    q = np.concatenate([keys, wl.distinct_keys(41, wl.MISS_INDEX_BASE, 1000)])
    for ts in (*snaps, mv.LATEST):
        assert np.array_equal(find(torch, t, q, ts), find(torch, c, q, ts)), f"snapshot {ts}"
    assert t.validate_tree_structure()["key_checksum"] == c.validate_tree_structure()["key_checksum"]
    more = wl.distinct_keys(41, 1 << 20, 5000)
    c.insert(dev(torch, more), dev(torch, wl.values_for(more, 7)))
    assert np.all(find(torch, t, more, mv.LATEST) == 0xFFFFFFFF)
    assert np.array_equal(find(torch, c, more, mv.LATEST), wl.values_for(more, 7))
    assert t.check_errors() == 0 and c.check_errors() == 0


def test_saved_tree_loads_and_continues_identically(torch, tmp_path):
    import workload as wl
    import mvgpubtree_b200 as mv
    t, keys, snaps = build(torch, mv, wl, reclaim=True)
    path = tmp_path / "tree.mvbt"
    t.save(path)
    u = mv.load(path)
    assert isinstance(u, mv.gpu_versioned_btree)
    for ts in (*snaps, mv.LATEST):
        assert np.array_equal(find(torch, t, keys, ts), find(torch, u, keys, ts)), f"snapshot {ts}"
    # both continue from the same state: same snapshot ids, same results
    more = wl.distinct_keys(41, 1 << 21, 3000)
    for x in (t, u):
        x.insert(dev(torch, more), dev(torch, wl.values_for(more, 9)))
        x.reclaim()
    assert t.take_snapshot() == u.take_snapshot()
    q = np.concatenate([keys, more])
    assert np.array_equal(find(torch, t, q, mv.LATEST), find(torch, u, q, mv.LATEST))
    with pytest.raises(mv.MVBTError):
        mv.load(tmp_path / "missing.mvbt")


def test_launch_shapes_give_identical_batch_results(torch):
    import workload as wl
    import mvgpubtree_b200 as mv
    initial, seed = 200_000, 17
    init = wl.distinct_keys(seed, 0, initial)
    base = mv.gpu_versioned_btree(pool_bytes=1 << 30)
    base.insert(dev(torch, init), dev(torch, wl.values_for(init, 0)))
    gen = wl.MixGenerator(seed, initial, stride=wl.stride_for(initial), batch_median=4096.0,
                          batch_min=256, batch_max=32768)
    steps = [gen.generate(24) for _ in range(2)]
    outs = {}
    for shape in ((8, 0), (8, 4), (8, 6), (8, 8), (16, 0), (16, 4), (16, 6), (16, 8)):
        c = base.clone()
        p = c.batch_plan(max(b.num_ops for b in steps), 24)
        p.set_launch(*shape)
        got = []
        for b in steps:
            res = torch.empty(b.num_ops, dtype=torch.int32, device="cuda")
            rout = torch.full((max(1, b.range_pairs) * 2,), -1, dtype=torch.int32, device="cuda")
            p.run(b.batch_off, dev(torch, b.type), dev(torch, b.key), dev(torch, b.arg),
                  dev(torch, b.out_off), dev(torch, b.range_cap), res, rout)
            got.append((host(res).copy(), host(rout).copy()))
        assert c.check_errors() == 0
        outs[shape] = got
    ref = outs[(8, 0)]
    for shape, got in outs.items():
        for (r, o), (er, eo) in zip(got, ref):
            assert np.array_equal(r, er), shape
            assert np.array_equal(o, eo), shape
    with pytest.raises(mv.MVBTError):
        base.batch_plan(16, 1).set_launch(12, 0)


def test_autotune_leaves_the_tree_and_sets_the_plan(torch):
    import workload as wl
    from mvgpubtree_b200.autotune import autotune_batches, DEFAULT_CANDIDATES
    import mvgpubtree_b200 as mv
    initial, seed = 200_000, 23
    init = wl.distinct_keys(seed, 0, initial)
    t = mv.gpu_versioned_btree(pool_bytes=1 << 30)
    t.insert(dev(torch, init), dev(torch, wl.values_for(init, 0)))
    before = t.validate_tree_structure()
    gen = wl.MixGenerator(seed, initial, stride=wl.stride_for(initial), batch_median=4096.0,
                          batch_min=256, batch_max=32768)
    steps = [gen.generate(16) for _ in range(2)]
    plan = t.batch_plan(max(b.num_ops for b in steps), 16)
    tune = autotune_batches(t, steps, plan=plan)
    assert (tune["tile_width"], tune["blocks_per_sm"]) in DEFAULT_CANDIDATES
    assert len(tune["kernel_ms"]) == len(DEFAULT_CANDIDATES)
    assert plan.launch == (tune["tile_width"], tune["blocks_per_sm"])
    after = t.validate_tree_structure()
    assert after["key_checksum"] == before["key_checksum"] and after["nodes_allocated"] == before["nodes_allocated"]
