"""CPU tier: the oracle against the reference's known-answer tests and its own invariants."""
import numpy as np
import pytest

from cases import OracleDriver, load_cases, replay


@pytest.fixture(scope="module")
def golden():
    return load_cases()


def _case_params():
    _, index = load_cases()
    out = []
    for c in index:
        for kind in c["kinds"]:
            out.append(pytest.param(c["name"], kind, id=f"{c['name']}-{kind}"))
    return out


@pytest.mark.parametrize("name,kind", _case_params())
def test_oracle_matches_reference_known_answers(golden, name, kind):
    z, index = golden
    case = next(c for c in index if c["name"] == name)
    replay(OracleDriver(kind == "versioned"), z, case)


def test_oracle_snapshot_isolation_and_erase_versions():
    import oracle
    m = oracle.MVMap(True)
    m.insert([5, 6, 7], [50, 60, 70])
    s0 = m.take_snapshot()
    m.insert([5, 8], [55, 80])
    m.erase([6])
    s1 = m.take_snapshot()
    m.erase([7])
    assert list(m.find([5, 6, 7, 8], s0)) == [50, 60, 70, 0xFFFFFFFF]
    assert list(m.find([5, 6, 7, 8], s1)) == [55, 0xFFFFFFFF, 70, 80]
    assert list(m.find([5, 6, 7, 8])) == [55, 0xFFFFFFFF, 0xFFFFFFFF, 80]
    assert list(m.find([0])) == [0]  # root tombstone
    pairs, counts = m.range_query([1], [100], 8, s1)
    assert counts[0] == 3 and pairs[0, :3, 0].tolist() == [5, 7, 8]
    assert pairs[0, :3, 1].tolist() == [55, 70, 80]


def test_oracle_plain_tree_ignores_timestamps():
    import oracle
    m = oracle.MVMap(False)
    m.insert([1, 2], [10, 20])
    m.erase([1])
    assert list(m.find([1, 2], 0)) == [0xFFFFFFFF, 20]


def test_oracle_range_edges():
    import oracle
    m = oracle.MVMap(True)
    keys = np.arange(10, 110, 10, dtype=np.uint32)
    m.insert(keys, keys * 2)
    # empty (lo >= hi), clipped to cap, saturated upper bound, lower above every key
    pairs, counts = m.range_query([50, 10, 95, 200], [50, 0xFFFFFFFF, 0xFFFFFFFF, 300], 3)
    assert counts.tolist() == [0, 10, 1, 0]
    assert pairs[1, :, 0].tolist() == [10, 20, 30]
    assert pairs[2, 0].tolist() == [100, 200]


def test_batch_runner_matches_step_by_step_replay():
    """orc_run_batches == snapshot / reads / writes issued one call at a time."""
    import oracle
    import workload as wl
    seed, n0 = 11, 20000
    gen = wl.MixGenerator(seed, n0, stride=wl.stride_for(n0), batch_median=512, batch_min=64,
                          batch_max=4096)
    b = gen.generate(12)
    init = wl.distinct_keys(seed, 0, n0)
    a = oracle.MVMap(True)
    a.insert(init, wl.values_for(init, 0))
    a.take_snapshot()
    res, out = a.run_batches(b)
    m = oracle.MVMap(True)
    m.insert(init, wl.values_for(init, 0))
    m.take_snapshot()
    for i in range(b.num_batches):
        lo, hi = int(b.batch_off[i]), int(b.batch_off[i + 1])
        t, k, g = b.type[lo:hi], b.key[lo:hi], b.arg[lo:hi]
        s = m.epoch
        f = t == wl.OP_FIND
        assert np.array_equal(m.find(k[f], s), res[lo:hi][f])
        r = np.nonzero(t == wl.OP_RANGE)[0]
        for j in r:
            cap = int(b.range_cap[lo + j])
            pairs, counts = m.range_query(k[j:j + 1], g[j:j + 1], cap, s)
            assert counts[0] == res[lo + j]
            c = min(int(counts[0]), cap)
            off = int(b.out_off[lo + j])
            assert np.array_equal(out[2 * off:2 * (off + c)].reshape(c, 2), pairs[0, :c])
        m.take_snapshot()
        m.insert(k[t == wl.OP_INSERT], g[t == wl.OP_INSERT])
        m.erase(k[t == wl.OP_ERASE])
    assert a.size() == m.size()


@pytest.mark.parametrize("parts", [1, 3, 8])
def test_partitioned_oracle_equals_sequential(parts):
    import oracle
    import workload as wl
    seed, n0 = 5, 50000
    gen = wl.MixGenerator(seed, n0, stride=wl.stride_for(n0) * 8, batch_median=2000)
    b = gen.generate(16)
    init = wl.distinct_keys(seed, 0, n0)
    a = oracle.MVMap(True)
    a.insert(init, wl.values_for(init, 0))
    p = oracle.PartitionedMVMap(parts, True)
    p.insert(init, wl.values_for(init, 0))
    r1, o1 = a.run_batches(b)
    r2, o2 = p.run_batches(b)
    assert np.array_equal(r1, r2)
    assert np.array_equal(o1, o2)
