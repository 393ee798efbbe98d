"""The oracle's per-query restatements agree with the plan oracle (itself pinned to the reference's
known answers) on the same seeded tables, and the generators are deterministic."""
import numpy as np
import pytest

from vectisdb_b200 import workloads as W
from vectisdb_b200.engine import hugeint_to_int
from oracle import oracle as O
from oracle.plan_oracle import evaluate


def _by_key(cols, nkeys):
    keys = list(zip(*[c.data.tolist() for c in cols[:nkeys]]))
    order = sorted(range(len(keys)), key=lambda i: keys[i])
    return [[c.data[i] for i in order] for c in cols]


def test_c0_oracle_matches_plan_oracle():
    wl = W.c0(n=200_000)
    k, v, w = [c.data for c in wl.inputs]
    exp = O.c0(k, v, w, 0.5, 7)
    got = _by_key(evaluate(wl.plan, wl.inputs), 1)
    assert np.array_equal(exp["k"], got[0])
    assert np.allclose(exp["sum"], got[1], rtol=1e-12, atol=0)
    assert np.array_equal(exp["count"], got[2])
    assert np.array_equal(exp["min"], got[3]) and np.array_equal(exp["max"], got[4])


def test_c1_oracle_matches_plan_oracle():
    wl = W.c1(n=30_000)
    a, b, amt, v, ts = [c.data for c in wl.inputs]
    exp = O.c1(a, b, amt, v, ts, wl.params["ts_gt"])
    cols = evaluate(wl.plan, wl.inputs)
    got = _by_key(cols, 2)
    assert np.array_equal(exp["a"], got[0]) and np.array_equal(exp["b"], got[1])
    sums = [int(h) * (1 << 64) + int(lo) for lo, h in zip(exp["sum_lo"], exp["sum_hi"])]
    assert sums == [int(x["upper"]) * (1 << 64) + int(x["lower"]) for x in got[2]]
    assert np.allclose(exp["avg"], got[3], rtol=1e-12, atol=0)
    assert np.array_equal(exp["count"], got[4]) and np.array_equal(exp["max"], got[5])


def test_c2_oracle_matches_plan_oracle():
    wl = W.c2(probe_n=50_000, build_n=4096, miss_lo=4096, miss_span=4096)
    pkey, x, bkey, g = [c.data for c in wl.inputs]
    exp = O.c2(bkey, g, pkey, x)
    got = _by_key(evaluate(wl.plan, wl.inputs), 1)
    assert np.array_equal(exp["g"], got[0])
    assert np.allclose(exp["sum"], got[1], rtol=1e-12, atol=0)


def test_c2b_oracle_matches_plan_oracle():
    wl = W.c2b(side=300)
    a, b = [c.data for c in wl.inputs]
    count, ea, eb = O.c2b(a, b, 13)
    got = evaluate(wl.plan, wl.inputs)
    assert count == len(got[0].data)
    assert np.array_equal(ea, got[0].data) and np.array_equal(eb, got[1].data)


def test_generators_are_deterministic_and_prefix_stable():
    a = W.uniform_i64(7, 3, 1000, 0, 1 << 62)
    b = W.uniform_i64(7, 3, 600, 0, 1 << 62)
    c = W.uniform_i64(7, 3, 400, 0, 1 << 62, offset=600)
    assert np.array_equal(a[:600], b) and np.array_equal(a[600:], c)
    assert not np.array_equal(a, W.uniform_i64(8, 3, 1000, 0, 1 << 62))
    z = W.zipf_i32(1, 0, 200_000, 1 << 20, 1.1)
    top = np.bincount(z)[:3] / len(z)
    assert 0.10 < top[0] < 0.15 and top[0] > top[1] > top[2]  # P(rank 1) ~ 0.124 for s=1.1 over 2^20
    p = W.permutation_i64(2, 0, 10_000)
    assert np.array_equal(np.sort(p), np.arange(10_000))
    u = W.uniform_f64(0, 1, 100_000)
    assert 0.0 <= u.min() and u.max() < 1.0 and abs(u.mean() - 0.5) < 0.01


def test_c1_shapes_match_the_configuration():
    wl = W.c1(n=1 << 16)
    a, b, amt, v, ts = [c.data for c in wl.inputs]
    assert a.min() >= 0 and a.max() < (1 << 20) and b.min() >= 0 and b.max() < 16
    assert amt.min() >= 0 and amt.max() < 1_000_000 and ts.min() >= 0
    med = wl.params["ts_gt"]
    assert np.sum(ts <= med) == (len(ts) - 1) // 2 + 1  # lower median


def test_c2_probe_hit_fraction():
    wl = W.c2(probe_n=100_000, build_n=1 << 14, miss_lo=1 << 14, miss_span=1 << 14)
    pkey = wl.inputs[0].data
    hits = np.mean(pkey < (1 << 14))
    assert 0.88 < hits < 0.92


def test_c2_oracle_with_repeated_build_keys_matches_plan_oracle():
    """Build keys that repeat (each key twice, some three times): every probe row pairs with every equal
    build row, as DuckDB's join does."""
    wl = W.c2(probe_n=40_000, build_n=2048, miss_lo=2048, miss_span=2048)
    pkey, x, bkey, g = [c.data for c in wl.inputs]
    rng = np.random.default_rng(8)
    bkey2 = np.concatenate([bkey, bkey, bkey[:300]])
    g2 = rng.integers(0, 64, len(bkey2)).astype(np.int32)
    exp = O.c2(bkey2, g2, pkey, x)
    from vectisdb_b200.engine import GpuValueType as T, make_column
    got = _by_key(evaluate(wl.plan, [make_column("pkey", T.INT64, pkey), make_column("x", T.FLOAT64, x),
                                     make_column("bkey", T.INT64, bkey2), make_column("g", T.INT32, g2)]), 1)
    assert np.array_equal(exp["g"], got[0])
    assert np.allclose(exp["sum"], got[1], rtol=1e-12, atol=0)


def test_cp_oracle_matches_plan_oracle():
    wl = W.cp(n=100_000)
    k, v, w = [c.data for c in wl.inputs]
    exp = O.cp(k, v, w, 0.5, 7)
    got = evaluate(wl.plan, wl.inputs)
    assert len(got[0].data) == len(exp["k"]) > 0
    assert np.array_equal(exp["k"], got[0].data)
    assert np.array_equal(exp["v"], got[1].data)  # v*2+1 rounds twice on both sides: bit-exact
    assert np.array_equal(exp["w"], got[2].data)
