"""GPU tier: the serving loop (mvbt_serve_trace), continuous batching over the persistent path.

A trace of mixed requests with Poisson arrivals is served with several requests per launch and
reclamation between launches. Every request's results must be
  * the oracle's for that request applied after all earlier requests (bit-exact), and
  * the same as the request run alone, in the same order, on an identical tree (one batch per
    launch), and as in the plain mode with one request per launch.
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


def range_views(b, result, range_out):
    """(op index, count, first min(count, cap) pairs) of every range query, for comparisons that
    ignore the unspecified rest of each slot."""
    out = []
    for i in np.nonzero(b.type == 3)[0]:
        c = int(result[i])
        m = min(c, int(b.range_cap[i]))
        o = int(b.out_off[i])
        out.append((int(i), c, range_out[o:o + m].tobytes()))
    return out


def make_tree(torch, mv, wl, initial, seed, w, reclaim):
    t = mv.gpu_versioned_btree(pool_bytes=1 << 30, tile_width=w, reclaim=reclaim)
    init = wl.distinct_keys(seed, 0, initial)
    t.insert(dev(torch, init), dev(torch, wl.values_for(init, 0)))
    return t, init


@pytest.mark.parametrize("w", [8, 16])
def test_served_requests_match_oracle_and_alone(torch, w):
    from mvgpubtree_b200 import workload as wl
    import mvgpubtree_b200 as mv
    import oracle
    initial, seed, R = 100_000, 77, 1200
    b, arrival = wl.serving_trace(seed, initial, R, offered_mops=20.0, stride=wl.stride_for(initial),
                                  batch_max=8192)
    t, init = make_tree(torch, mv, wl, initial, seed, w, reclaim=True)
    out = t.serve(b, arrival, reclaim_every=4, max_requests_per_launch=64)
    assert t.check_errors() == 0
    st = out["stats"]
    assert st["requests"] == R and st["ops"] == b.num_ops
    assert st["launches"] < R, st  # several requests per launch
    assert st["reclaims"] > 0 and t.stats()["reclaimed"] > 0
    snaps = out["snapshot"].astype(np.int64)
    assert np.all(np.diff(snaps) == 1)  # one snapshot per request, in order
    assert np.all(out["done_ns"] >= arrival)
    served = range_views(b, out["result"], out["range_out"])
    find = b.type == 0
    # the oracle: each request applied after all earlier ones
    m = oracle.MVMap(True)
    m.insert(init, wl.values_for(init, 0))
    er, eo = m.run_batches(b)
    assert np.array_equal(out["result"][find], er[find])
    assert served == range_views(b, er, eo.reshape(-1, 2))
    # each request alone, one launch each, same order, on an identical tree
    a, _ = make_tree(torch, mv, wl, initial, seed, w, reclaim=False)
    plan = a.batch_plan(int(np.diff(b.batch_off.astype(np.int64)).max()) + 1, 1)
    res = np.zeros(b.num_ops, np.uint32)
    rout = np.full((max(1, b.range_pairs), 2), 0xFFFFFFFF, np.uint32)
    for r in range(R):
        lo, hi = int(b.batch_off[r]), int(b.batch_off[r + 1])
        if hi == lo:
            continue
        rq = b.type[lo:hi] == 3
        base = int(b.out_off[lo:hi][rq].min()) if rq.any() else 0
        ro = np.where(rq, b.out_off[lo:hi] - np.uint64(base), 0).astype(np.uint64)
        pairs = max(8, int((ro[rq] + b.range_cap[lo:hi][rq]).max())) if rq.any() else 8
        r_res = torch.empty(hi - lo, dtype=torch.int32, device="cuda")
        r_out = torch.full((pairs * 2,), -1, dtype=torch.int32, device="cuda")
        plan.run(np.array([0, hi - lo], np.uint64), dev(torch, b.type[lo:hi]), dev(torch, b.key[lo:hi]),
                 dev(torch, b.arg[lo:hi]), dev(torch, ro.astype(np.uint64)), dev(torch, b.range_cap[lo:hi]),
                 r_res, r_out, mode=mv.BATCH_PERSISTENT)
        res[lo:hi] = host(r_res)
        rr = host(r_out).reshape(-1, 2)
        for i in np.nonzero(rq)[0]:
            o, c = int(ro[i]), int(b.range_cap[lo + i])
            rout[base + o: base + o + c] = rr[o:o + c]
    assert a.check_errors() == 0
    assert np.array_equal(out["result"][find], res[find])
    assert served == range_views(b, res, rout)
    # the plain mode, one request per launch, on an identical tree
    p, _ = make_tree(torch, mv, wl, initial, seed, w, reclaim=False)
    plain = p.serve(b, arrival, mode=mv.BATCH_PER_LAUNCH)
    assert plain["stats"]["launches"] == np.count_nonzero(np.diff(b.batch_off.astype(np.int64)))
    bad = np.nonzero(find & (plain["result"] != out["result"]))[0]
    assert bad.size == 0, (
        f"{bad.size} finds differ in the plain mode; first: "
        + ", ".join(f"op {i} key {int(b.key[i]):#x} plain {int(plain['result'][i]):#x} "
                    f"served {int(out['result'][i]):#x} oracle {int(er[i]):#x}" for i in bad[:4]))
    assert range_views(b, plain["result"], plain["range_out"]) == served


def test_serving_rejects_bad_traces(torch):
    from mvgpubtree_b200 import workload as wl
    import mvgpubtree_b200 as mv
    b, arrival = wl.serving_trace(5, 1000, 20, offered_mops=1.0, stride=wl.stride_for(1000))
    t = mv.gpu_versioned_btree(pool_bytes=1 << 26)
    with pytest.raises(mv.MVBTError):
        t.serve(b, arrival[::-1].copy())  # arrivals must not decrease
    with pytest.raises(mv.MVBTError):
        t.serve(b, arrival, reclaim_every=1)  # the tree was made without reclaim
    with pytest.raises(mv.MVBTError):
        t.serve(b, arrival, max_ops_per_launch=1)  # a request is larger than a launch
