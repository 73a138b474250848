"""GPU tier: mixed batches through the entry point that allocates nothing.

mvbt_batch_run_noalloc is for callers that cannot allocate device memory on their call path --
a serving loop with a latency budget, where cudaMalloc / cudaFree could block the device, or a
host that owns every allocation and gives the library a fixed budget. Its scratch is a fixed
array inside the library. This test calls it through the C ABI twice in a row and checks every
result against the plan-based entry point (mvbt_batch_run, persistent mode) running the same
batches on an identical tree. The work is integer and bit-exact, so the tolerance is zero.
The file name makes pytest collect it last.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need CUDA"
    return t


def _dev(torch, a):
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        return torch.from_numpy(a.view(np.int64)).cuda()
    return torch.from_numpy(a.astype(np.uint32, copy=False).view(np.int32)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint32)


def test_noalloc_batches_match_plan_batches_twice(torch):
    import mvgpubtree_b200 as mv
    import workload as wl
    seed, n0 = 77, 1 << 17
    init = wl.distinct_keys(seed, 0, n0)
    vals = wl.values_for(init, 0)
    trees = []
    for _ in range(2):
        t = mv.gpu_versioned_btree(pool_bytes=1 << 30)
        t.insert(_dev(torch, init), _dev(torch, vals))
        trees.append(t)
    plan = trees[0].batch_plan(mv.NOALLOC_MAX_OPS, mv.NOALLOC_MAX_BATCHES)
    gen = wl.MixGenerator(seed, n0, stride=wl.stride_for(n0), batch_median=2048, batch_max=1 << 15)
    for call in range(2):  # two calls in a row: the shared array must start clean every time
        b = gen.generate(40)
        assert b.num_ops <= mv.NOALLOC_MAX_OPS
        ops = [_dev(torch, b.type), _dev(torch, b.key), _dev(torch, b.arg), _dev(torch, b.out_off),
               _dev(torch, b.range_cap)]
        outs = []
        for k, t in enumerate(trees):
            result = torch.zeros(b.num_ops, dtype=torch.int32, device="cuda")
            rout = torch.full((max(1, b.range_pairs) * 2,), -1, dtype=torch.int32, device="cuda")
            if k == 0:
                plan.run(b.batch_off, *ops, result, rout, mode=mv.BATCH_PERSISTENT)
            else:
                t.batch_run_noalloc(_dev(torch, b.batch_off), b.num_ops, *ops, result, rout)
            t.check_errors()
            outs.append((_host(result), _host(rout)))
        assert np.array_equal(outs[0][0], outs[1][0]), f"call {call}: results differ"
        assert np.array_equal(outs[0][1], outs[1][1]), f"call {call}: range outputs differ"
    r0, r1 = (t.validate_tree_structure() for t in trees)
    assert r0["keys"] == r1["keys"] and r0["key_checksum"] == r1["key_checksum"]
    assert trees[0].take_snapshot() == trees[1].take_snapshot()


def test_noalloc_rejects_requests_beyond_its_limits(torch):
    import mvgpubtree_b200 as mv
    t = mv.gpu_versioned_btree(pool_bytes=1 << 26)
    z = torch.zeros(4, dtype=torch.int32, device="cuda")
    off = torch.zeros(mv.NOALLOC_MAX_BATCHES + 2, dtype=torch.int64, device="cuda")
    with pytest.raises(mv.MVBTError, match="MVBT_NOALLOC_MAX_BATCHES"):
        t.batch_run_noalloc(off, 0, z, z, z, off, z, z, off)
    off2 = torch.zeros(2, dtype=torch.int64, device="cuda")
    with pytest.raises(mv.MVBTError, match="MVBT_NOALLOC_MAX_OPS"):
        t.batch_run_noalloc(off2, mv.NOALLOC_MAX_OPS + 1, z, z, z, off2, z, z, off2)
    assert t.check_errors() == 0


def test_noalloc_rejects_offsets_of_the_wrong_width(torch):
    """batch_off and out_off are read as 64-bit words: a 32-bit or floating-point tensor is turned
    away on the host before any kernel could read past its end."""
    import mvgpubtree_b200 as mv
    t = mv.gpu_versioned_btree(pool_bytes=1 << 26)
    z = torch.zeros(4, dtype=torch.int32, device="cuda")
    off = torch.tensor([0, 4], dtype=torch.int64, device="cuda")
    for bad in (torch.tensor([0, 4], dtype=torch.int32, device="cuda"),
                torch.tensor([0.0, 4.0], dtype=torch.float64, device="cuda")):
        with pytest.raises(TypeError, match="batch_off"):
            t.batch_run_noalloc(bad, 4, z, z, z, off, z, z, off)
        with pytest.raises(TypeError, match="out_off"):
            t.batch_run_noalloc(off, 4, z, z, z, bad, z, z, off)
    assert t.check_errors() == 0


def test_noalloc_rejects_bad_offsets_on_the_device(torch):
    """Offsets that do not start at 0, decrease, or end elsewhere than num_ops are caught by the
    device-side check: nothing runs (results and the tree stay as they were) and the tree reports
    MVBT_ERR_CORRUPT from the check's own error site."""
    import mvgpubtree_b200 as mv
    import workload as wl
    seed, n0 = 91, 1 << 14
    init = wl.distinct_keys(seed, 0, n0)
    t = mv.gpu_versioned_btree(pool_bytes=1 << 27)
    t.insert(_dev(torch, init), _dev(torch, wl.values_for(init, 0)))
    before = t.validate_tree_structure()
    gen = wl.MixGenerator(seed, n0, stride=wl.stride_for(n0), batch_median=256, batch_min=64, batch_max=1024)
    b = gen.generate(4)
    ops = [_dev(torch, b.type), _dev(torch, b.key), _dev(torch, b.arg), _dev(torch, b.out_off),
           _dev(torch, b.range_cap)]
    n = b.num_ops
    good = b.batch_off.astype(np.int64)
    cases = {"decreasing": np.array([0, good[2], good[1], good[3], n], np.int64),
             "wrong_end": np.array([0, good[1], good[2], good[3], n - 1], np.int64),
             "nonzero_start": np.array([1, good[1], good[2], good[3], n], np.int64)}
    for name, off in cases.items():
        site0 = t.stats()["error_sites"].get(16, 0)
        result = torch.full((n,), 7, dtype=torch.int32, device="cuda")
        rout = torch.full((max(1, b.range_pairs) * 2,), 7, dtype=torch.int32, device="cuda")
        t.batch_run_noalloc(torch.from_numpy(off).cuda(), n, *ops, result, rout)
        bits = t.check_errors(raise_on_error=False)
        assert bits & 4, f"{name}: expected MVBT_ERR_CORRUPT, got bits {bits}"
        assert t.stats()["error_sites"].get(16, 0) == site0 + 1, name
        t.clear_errors()
        assert bool((result == 7).all()) and bool((rout == 7).all()), f"{name}: a kernel wrote results"
        after = t.validate_tree_structure()
        assert (after["keys"], after["key_checksum"]) == (before["keys"], before["key_checksum"]), name
    assert t.check_errors() == 0
    t.close()
