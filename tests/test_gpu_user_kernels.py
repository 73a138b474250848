"""GPU tier: user kernels written against the reference's device API names.

tests/cpp/user_kernels.cu holds kernels written the way a reference user writes them -- one key
per thread, each tile of 8 or 16 threads serving its threads' keys through
tree.cooperative_insert / cooperative_erase / cooperative_find / concurrent_cooperative_range_query /
cooperative_range_query / take_snapshot with an allocator context -- compiled against include/
(gpu_btree_device.cuh over mvbt_device.cuh) and given the tree through the C ABI's device view.
Their results must equal the oracle's, on both tree kinds and both tile widths.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need CUDA"
    return t


@pytest.fixture(scope="module")
def uk():
    import mvgpubtree_b200  # noqa: F401  (loads libmvbt.so first: the kernels link against it)
    from pathlib import Path
    so = Path(__file__).resolve().parent / "cpp" / "libuser_kernels.so"
    lib = ctypes.CDLL(str(so))
    vp, u32, i = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int
    for name, args in {"uk_insert": [vp, i, i, vp, vp, u32], "uk_erase": [vp, i, i, vp, u32],
                       "uk_find": [vp, i, i, vp, vp, u32, u32, i],
                       "uk_range": [vp, i, i, vp, vp, vp, vp, u32, u32, u32],
                       "uk_take_snapshot": [vp, i, vp]}.items():
        f = getattr(lib, name)
        f.restype, f.argtypes = i, args
    return lib


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, np.uint32).view(np.int32)).cuda()


def host(t):
    return t.cpu().numpy().view(np.uint32)


def ptr(t):
    return t.data_ptr()


@pytest.mark.parametrize("w", [8, 16])
def test_user_kernels_on_the_versioned_tree_match_oracle(torch, uk, w):
    import mvgpubtree_b200 as mv
    import oracle
    import workload as wl
    seed, n0 = 71, 1 << 16
    keys = wl.distinct_keys(seed, 0, n0)
    vals = wl.values_for(keys, seed)
    t = mv.gpu_versioned_btree(pool_bytes=1 << 28)
    h = t.handle
    m = oracle.MVMap(True)
    dk, dv = dev(torch, keys), dev(torch, vals)
    assert uk.uk_insert(h, 1, w, ptr(dk), ptr(dv), n0) == 0
    m.insert(keys, vals)
    snap = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert uk.uk_take_snapshot(h, w, ptr(snap)) == 0
    s0 = int(host(snap)[0]); assert s0 == m.take_snapshot()
    upd = wl.shuffle(seed + 1, keys)[: n0 // 4]
    du, duv = dev(torch, upd), dev(torch, wl.values_for(upd, seed ^ 1))
    assert uk.uk_insert(h, 1, w, ptr(du), ptr(duv), upd.size) == 0
    m.insert(upd, wl.values_for(upd, seed ^ 1))
    er = wl.shuffle(seed + 2, keys)[: n0 // 5]
    de = dev(torch, er)
    assert uk.uk_erase(h, 1, w, ptr(de), er.size) == 0
    m.erase(er)
    assert uk.uk_take_snapshot(h, w, ptr(snap)) == 0
    s1 = int(host(snap)[0]); assert s1 == m.take_snapshot()
    assert t.check_errors() == 0
    q = wl.shuffle(seed + 3, np.concatenate([keys, wl.distinct_keys(seed, wl.MISS_INDEX_BASE, 4096)]))
    dq = dev(torch, q)
    out = torch.empty(q.size, dtype=torch.int32, device="cuda")
    for ts in (s0, s1, mv.LATEST):
        for concurrent in (0, 1):
            assert uk.uk_find(h, 1, w, ptr(dq), ptr(out), q.size, ts, concurrent) == 0
            assert np.array_equal(host(out), m.find(q, ts)), (ts, concurrent)
    nq, slot = 2048, 64
    lo = wl.uniform_keys(seed + 4, nq)
    hi = wl.upper_bounds(lo, 16, wl.stride_for(n0))
    pairs = torch.full((nq * slot * 2,), -1, dtype=torch.int32, device="cuda")
    counts = torch.zeros(nq, dtype=torch.int32, device="cuda")
    for ts in (s0, s1):
        ep, ec = m.range_query(lo, hi, slot, ts)
        assert int(ec.max()) <= slot  # the reference's contract: the slot holds every hit
        assert uk.uk_range(h, 1, w, ptr(dev(torch, lo)), ptr(dev(torch, hi)), ptr(pairs), ptr(counts), slot, nq, ts) == 0
        assert np.array_equal(host(counts), ec), ts
        gp = host(pairs).reshape(nq, slot, 2)
        mask = np.arange(slot)[None, :] < ec[:, None]
        assert np.array_equal(gp[mask], ep[mask]), ts
    assert t.check_errors() == 0
    rep = t.validate_tree_structure()
    assert rep["violations"] == 0 and rep["keys"] == m.size()


@pytest.mark.parametrize("w", [8, 16])
def test_user_kernels_on_the_blink_tree_match_oracle(torch, uk, w):
    import mvgpubtree_b200 as mv
    import oracle
    import workload as wl
    seed, n0 = 73, 1 << 16
    keys = wl.distinct_keys(seed, 0, n0)
    vals = wl.values_for(keys, seed)
    t = mv.gpu_blink_tree(pool_bytes=1 << 28)
    h = t.handle
    m = oracle.MVMap(False)
    assert uk.uk_insert(h, 0, w, ptr(dev(torch, keys)), ptr(dev(torch, vals)), n0) == 0
    m.insert(keys, vals)
    er = wl.shuffle(seed + 1, keys)[: n0 // 3]
    assert uk.uk_erase(h, 0, w, ptr(dev(torch, er)), er.size) == 0
    m.erase(er)
    q = wl.shuffle(seed + 2, np.concatenate([keys, wl.distinct_keys(seed, wl.MISS_INDEX_BASE, 4096)]))
    out = torch.empty(q.size, dtype=torch.int32, device="cuda")
    assert uk.uk_find(h, 0, w, ptr(dev(torch, q)), ptr(out), q.size, mv.LATEST, 1) == 0
    assert np.array_equal(host(out), m.find(q))
    nq, slot = 2048, 64
    lo = wl.uniform_keys(seed + 3, nq)
    hi = wl.upper_bounds(lo, 16, wl.stride_for(n0))
    pairs = torch.full((nq * slot * 2,), -1, dtype=torch.int32, device="cuda")
    counts = torch.zeros(nq, dtype=torch.int32, device="cuda")
    ep, ec = m.range_query(lo, hi, slot)
    assert uk.uk_range(h, 0, w, ptr(dev(torch, lo)), ptr(dev(torch, hi)), ptr(pairs), ptr(counts), slot, nq, mv.LATEST) == 0
    assert np.array_equal(host(counts), ec)
    mask = np.arange(slot)[None, :] < ec[:, None]
    assert np.array_equal(host(pairs).reshape(nq, slot, 2)[mask], ep[mask])
    assert t.check_errors() == 0
