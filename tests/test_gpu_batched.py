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
    from mvgpubtree_b200 import workload as wl
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
    from mvgpubtree_b200 import workload as wl
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
    from mvgpubtree_b200 import workload as wl
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
