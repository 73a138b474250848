"""GPU tier: the serving loop (mvbt_serve_trace), continuous batching over the persistent path.

A trace of mixed requests with Poisson arrivals is served with several requests per launch.
  * One snapshot per admitted batch (the default): requests admitted together share a snapshot.
    Their results must equal the oracle's with the same groups applied as batches, and each
    group's reads run alone afterwards at its snapshot must return the same results.
  * One snapshot per request: every request's results must equal the oracle's for that request
    applied after all earlier requests, the request run alone in the same order on an identical
    tree, and the plain mode with one request per launch.
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
def test_served_groups_match_oracle_and_alone_at_their_snapshot(torch, w):
    import workload as wl
    import mvgpubtree_b200 as mv
    import oracle
    initial, seed, R = 100_000, 91, 1500
    b, arrival = wl.serving_trace(seed, initial, R, offered_mops=40.0, stride=wl.stride_for(initial),
                                  batch_max=8192, erase_lag=128)
    t, init = make_tree(torch, mv, wl, initial, seed, w, reclaim=False)  # keep every snapshot
    out = t.serve(b, arrival, max_requests_per_launch=64)
    assert t.check_errors() == 0
    st = out["stats"]
    assert st["requests"] == R and st["launches"] < R, st
    snaps = out["snapshot"].astype(np.int64)
    steps = np.diff(snaps)
    assert np.all((steps == 0) | (steps == 1))  # groups in order, one snapshot each
    starts = np.concatenate([[0], np.nonzero(steps)[0] + 1, [R]])
    group_off = b.batch_off[starts].astype(np.uint64)
    served = range_views(b, out["result"], out["range_out"])
    find = b.type == 0
    # the oracle with the same groups applied as batches
    m = oracle.MVMap(True)
    m.insert(init, wl.values_for(init, 0))
    g = wl.Batches(group_off, b.type, b.key, b.arg, b.out_off, b.range_cap, b.range_pairs)
    er, eo = m.run_batches(g)
    assert np.array_equal(out["result"][find], er[find])
    assert served == range_views(b, er, eo.reshape(-1, 2))
    # each group's reads alone, afterwards, at the group's snapshot
    for k in range(len(starts) - 1):
        lo, hi = int(group_off[k]), int(group_off[k + 1])
        S = int(snaps[starts[k]])
        ty = b.type[lo:hi]
        fk = b.key[lo:hi][ty == 0]
        if fk.size:
            o = torch.empty(fk.size, dtype=torch.int32, device="cuda")
            t.find(dev(torch, fk), o, timestamp=S)
            assert np.array_equal(host(o), out["result"][lo:hi][ty == 0]), f"group {k} finds"
        rq = np.nonzero(ty == 3)[0]
        if rq.size:
            cap = int(b.range_cap[lo:hi][rq].max())
            pr = torch.full((rq.size * cap * 2,), -1, dtype=torch.int32, device="cuda")
            cn = torch.empty(rq.size, dtype=torch.int32, device="cuda")
            t.range_query(dev(torch, b.key[lo:hi][rq]), dev(torch, b.arg[lo:hi][rq]), pr, cn, cap,
                          rq.size, S)
            alone = host(pr).reshape(rq.size, cap, 2)
            counts = host(cn)
            for j, i in enumerate(rq):
                op = lo + int(i)
                c, m_ = int(counts[j]), min(int(counts[j]), int(b.range_cap[op]))
                o_ = int(b.out_off[op])
                assert c == int(out["result"][op]), f"group {k} range count"
                assert alone[j, :m_].tobytes() == out["range_out"][o_:o_ + m_].tobytes(), f"group {k} pairs"


@pytest.mark.parametrize("w", [8, 16])
def test_per_request_snapshots_match_oracle_and_alone(torch, w):
    import workload as wl
    import mvgpubtree_b200 as mv
    import oracle
    initial, seed, R = 100_000, 77, 1200
    b, arrival = wl.serving_trace(seed, initial, R, offered_mops=20.0, stride=wl.stride_for(initial),
                                  batch_max=8192, erase_lag=0)
    t, init = make_tree(torch, mv, wl, initial, seed, w, reclaim=True)
    out = t.serve(b, arrival, reclaim_every=4, max_requests_per_launch=64,
                  snapshots=mv.SERVE_SNAPSHOT_PER_REQUEST)
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
    plain = p.serve(b, arrival, mode=mv.BATCH_PER_LAUNCH, snapshots=mv.SERVE_SNAPSHOT_PER_REQUEST)
    assert plain["stats"]["launches"] == np.count_nonzero(np.diff(b.batch_off.astype(np.int64)))
    bad = np.nonzero(find & (plain["result"] != out["result"]))[0]
    assert bad.size == 0, (
        f"{bad.size} finds differ in the plain mode; first: "
        + ", ".join(f"op {i} key {int(b.key[i]):#x} plain {int(plain['result'][i]):#x} "
                    f"served {int(out['result'][i]):#x} oracle {int(er[i]):#x}" for i in bad[:4]))
    assert range_views(b, plain["result"], plain["range_out"]) == served


def test_serving_rejects_bad_traces(torch):
    import workload as wl
    import mvgpubtree_b200 as mv
    b, arrival = wl.serving_trace(5, 1000, 20, offered_mops=1.0, stride=wl.stride_for(1000))
    t = mv.gpu_versioned_btree(pool_bytes=1 << 26)
    with pytest.raises(mv.MVBTError):
        t.serve(b, arrival[::-1].copy())  # arrivals must not decrease
    with pytest.raises(mv.MVBTError):
        t.serve(b, arrival, reclaim_every=1)  # the tree was made without reclaim
    with pytest.raises(mv.MVBTError):
        t.serve(b, arrival, max_ops_per_launch=1)  # a request is larger than a launch


@pytest.mark.parametrize("w", [8, 16])
def test_serving_with_reclamation_inside_launches_and_lag_admission(torch, w):
    """Serving with reclamation inside every launch (reclaim_in_launch) and admission by
    reclamation lag (max_reclaim_lag): results are identical to the oracle with the same groups
    applied as batches, copies are freed and reused during the session, the lag limit defers
    admissions, and the node high-water mark stays below a session that keeps every version."""
    import workload as wl
    import mvgpubtree_b200 as mv
    import oracle
    initial, seed, R = 100_000, 93, 2000
    b, arrival = wl.serving_trace(seed, initial, R, offered_mops=40.0, stride=wl.stride_for(initial),
                                  batch_max=8192, erase_lag=128)
    outs, stats = {}, {}
    for name, kw in (("keep", {}), ("inside", {"reclaim_in_launch": 1, "max_reclaim_lag": 20000})):
        t, init = make_tree(torch, mv, wl, initial, seed, w, reclaim=bool(kw))
        outs[name] = t.serve(b, arrival, max_requests_per_launch=64, **kw)
        assert t.check_errors() == 0
        stats[name] = (outs[name]["stats"], t.stats(), t.compute_memory_usage()["nodes_allocated"])
        rep = t.validate_tree_structure()
        assert rep["violations"] == 0 and rep["locked_nodes"] == 0
    for name, out in outs.items():
        snaps = out["snapshot"].astype(np.int64)
        steps = np.diff(snaps)
        starts = np.concatenate([[0], np.nonzero(steps)[0] + 1, [R]])
        m = oracle.MVMap(True)
        m.insert(init, wl.values_for(init, 0))
        g = wl.Batches(b.batch_off[starts].astype(np.uint64), b.type, b.key, b.arg, b.out_off,
                       b.range_cap, b.range_pairs)
        er, eo = m.run_batches(g)
        find = b.type == 0
        assert np.array_equal(out["result"][find], er[find]), name
        assert range_views(b, out["result"], out["range_out"]) == range_views(b, er, eo.reshape(-1, 2)), name
    sv, tr, nodes = stats["inside"]
    assert tr["reclaimed"] > 0 and tr["reused"] > 0, tr
    assert sv["nodes_high_water"] > 0 and tr["log_dropped"] == 0
    assert nodes < stats["keep"][2], (nodes, stats["keep"][2])
