"""GPU tier: results identical to the reference implementation's own CUDA build on the same inputs.

oracle/_ref/ref_driver (built by oracle/ref_build.py from the reference's unmodified headers) runs
the reference through its public host API; this library runs the same workload through its C ABI;
checksums of every find result, range count and range pair are compared (tests/refbuild.py).
  * C1 shape: plain B-link tree, insert then finds (half present, half never inserted).
  * C4 shape: versioned tree, mixed batches with one snapshot per batch. The reference issues each
    batch in its plain form (take_snapshot, find(ts), range_query(ts), insert, erase); this library
    runs all batches in one persistent launch. A final snapshot reads the whole key space.
"""
import numpy as np
import pytest

from refbuild import DRIVER, find_sum, count_sum, pairs_sum, run_driver, step_sums

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
    from mvgpubtree_b200 import workload as wl
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
    from mvgpubtree_b200 import workload as wl
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
