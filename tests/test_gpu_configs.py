"""Parity of the benchmark queries: the engine (C ABI) against the oracle on the same seeded tables.

Integer, DECIMAL (exact 128-bit) and COUNT results must be bit-exact; DOUBLE sums and averages are
order-dependent FP64 and must agree within 1e-12 relative (the tolerance the query contract states).
"""
import numpy as np
import pytest

from vectisdb_b200 import GpuEngine
from vectisdb_b200 import workloads as W
from vectisdb_b200.engine import hugeint_to_int
from oracle import oracle as O

pytestmark = pytest.mark.gpu

REL = 1e-12


def _run(wl):
    r = GpuEngine.instance().execute_plan(wl.plan, wl.inputs)
    assert r.success, r.error_message
    return r.columns


def _close(got, exp):
    got = np.asarray(got, np.float64)
    exp = np.asarray(exp, np.float64)
    return np.all(np.abs(got - exp) <= REL * np.maximum(np.abs(exp), 1e-300))


@pytest.mark.parametrize("n,k_card", [(1 << 16, 1024), (1_000_003, 1024), (1 << 20, 16), (300_000, 3000)])
def test_c0_filter_group_by(n, k_card):
    wl = W.c0(n=n, k_card=k_card)
    cols = _run(wl)
    k, s, c, mn, mx = [x.data for x in cols]
    order = np.argsort(k)
    exp = O.c0(wl.inputs[0].data, wl.inputs[1].data, wl.inputs[2].data, 0.5, 7)
    assert np.array_equal(k[order], exp["k"])
    assert np.array_equal(c[order], exp["count"])
    assert np.array_equal(mn[order], exp["min"])
    assert np.array_equal(mx[order], exp["max"])
    assert _close(s[order], exp["sum"])


@pytest.mark.parametrize("n", [1 << 14, 1 << 18, 3_000_001])
def test_c1_high_cardinality_group_by(n):
    wl = W.c1(n=n)
    a, b, amt, v, ts = [c.data for c in wl.inputs]
    cols = _run(wl)
    ga, gb, gsum, gavg, gcnt, gmax = [c.data for c in cols]
    order = np.lexsort((gb, ga))
    exp = O.c1(a, b, amt, v, ts, wl.params["ts_gt"])
    assert len(ga) == len(exp["a"])
    assert np.array_equal(ga[order], exp["a"]) and np.array_equal(gb[order], exp["b"])
    assert np.array_equal(gcnt[order], exp["count"])
    assert np.array_equal(gmax[order], exp["max"])
    gs = gsum[order]
    assert np.array_equal(gs["lower"], exp["sum_lo"]) and np.array_equal(gs["upper"], exp["sum_hi"])
    assert _close(gavg[order], exp["avg"])


def test_c1_sum_is_exact_beyond_int64():
    """SUM over BIGINT returns HUGEINT: sums that overflow 64 bits stay exact (DuckDB's DECIMAL(38,x))."""
    from vectisdb_b200.engine import GpuAggregateKind as A, GpuValueType as T
    from vectisdb_b200 import make_aggregate, make_column, make_group_by, make_scan
    n = 1 << 16
    k = np.arange(n) % 3
    big = np.full(n, (1 << 62) + 12345, np.int64)
    big[::5] = -(1 << 62) - 7
    plan = make_group_by(["k"], [make_aggregate(A.SUM, "v", T.HUGEINT)], make_scan(["k", "v"]))
    r = GpuEngine.instance().execute_plan(plan, [make_column("k", T.INT32, k), make_column("v", T.INT64, big)])
    assert r.success, r.error_message
    got = dict(zip(r.columns[0].data.tolist(), hugeint_to_int(r.columns[1].data)))
    for key in range(3):
        assert got[key] == int(big[k == key].astype(object).sum())


@pytest.mark.parametrize("probe_n,build_n", [(1 << 16, 1 << 12), (1 << 20, 1 << 16)])
def test_c2_join_group_by(probe_n, build_n):
    wl = W.c2(probe_n=probe_n, build_n=build_n, miss_lo=build_n, miss_span=build_n)
    pkey, x, bkey, g = [c.data for c in wl.inputs]
    cols = _run(wl)
    gg, gs = [c.data for c in cols]
    order = np.argsort(gg)
    exp = O.c2(bkey, g, pkey, x)
    assert np.array_equal(gg[order], exp["g"])
    assert _close(gs[order], exp["sum"])


@pytest.mark.parametrize("side", [256, 1000, 4096])
def test_c2b_filtered_cross_product(side):
    wl = W.c2b(side=side)
    a, b = [c.data for c in wl.inputs]
    cols = _run(wl)
    count, ea, eb = O.c2b(a, b, 13)
    assert len(cols[0].data) == count
    assert np.array_equal(cols[0].data, ea) and np.array_equal(cols[1].data, eb)  # left-major order


@pytest.mark.parametrize("tier1,retry", [("256", None), ("256", "64")])
def test_c1_overflow_tiers_stay_exact(tier1, retry, monkeypatch):
    """Tables far too small for their partitions: tier-1 overflows go to the device retry list, and
    (with a tiny retry table too) on to the global-memory pass; the answer must not change."""
    monkeypatch.setenv("VGPU_GB_TABLE_SLOTS", tier1)
    if retry:
        monkeypatch.setenv("VGPU_GB_RETRY_SLOTS", retry)
    monkeypatch.setenv("VGPU_GB_PARTITIONS", "64")
    wl = W.c1(n=1 << 18)
    a, b, amt, v, ts = [c.data for c in wl.inputs]
    cols = _run(wl)
    ga, gb, gsum, gavg, gcnt, gmax = [c.data for c in cols]
    order = np.lexsort((gb, ga))
    exp = O.c1(a, b, amt, v, ts, wl.params["ts_gt"])
    assert np.array_equal(ga[order], exp["a"]) and np.array_equal(gb[order], exp["b"])
    assert np.array_equal(gcnt[order], exp["count"]) and np.array_equal(gmax[order], exp["max"])
    gs = gsum[order]
    assert np.array_equal(gs["lower"], exp["sum_lo"]) and np.array_equal(gs["upper"], exp["sum_hi"])
    assert _close(gavg[order], exp["avg"])


@pytest.mark.parametrize("n,env", [
    (1 << 14, {}),
    (1 << 18, {}),
    (3_000_001, {}),
    (1 << 18, {"VGPU_GB_SPLIT_ROWS": "256"}),             # most partitions split into merged chunks
    (1 << 18, {"VGPU_GB_DIRECT_BITS": "8"}),              # narrow tables, many partitions
    (1 << 18, {"VGPU_GB_DIRECT_BITS": "8", "VGPU_GB_SPLIT_ROWS": "256", "VGPU_GB_BUCKET_THREADS": "128"}),
])
def test_c1_direct_partitioned_strategy(n, env, monkeypatch):
    """The direct-partitioned strategy (bijective key mix, dense shared tables, split partitions merged
    through global tables) gives the same groups and aggregates as the oracle."""
    monkeypatch.setenv("VGPU_GB_STRATEGY", "direct")
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    wl = W.c1(n=n)
    a, b, amt, v, ts = [c.data for c in wl.inputs]
    cols = _run(wl)
    ga, gb, gsum, gavg, gcnt, gmax = [c.data for c in cols]
    order = np.lexsort((gb, ga))
    exp = O.c1(a, b, amt, v, ts, wl.params["ts_gt"])
    assert len(ga) == len(exp["a"])
    assert np.array_equal(ga[order], exp["a"]) and np.array_equal(gb[order], exp["b"])
    assert np.array_equal(gcnt[order], exp["count"]) and np.array_equal(gmax[order], exp["max"])
    gs = gsum[order]
    assert np.array_equal(gs["lower"], exp["sum_lo"]) and np.array_equal(gs["upper"], exp["sum_hi"])
    assert _close(gavg[order], exp["avg"])


@pytest.mark.parametrize("split", [None, "256"])
def test_direct_partitioned_signed_sums_and_min(split, monkeypatch):
    """Negative and beyond-64-bit integer sums through the 32-bit-word accumulators, plus MIN/MAX and
    FP64 sums, on a key space wide enough to need several partitions."""
    from vectisdb_b200.engine import GpuAggregateKind as A, GpuValueType as T
    from vectisdb_b200 import make_aggregate, make_column, make_group_by, make_scan
    monkeypatch.setenv("VGPU_GB_STRATEGY", "direct")
    monkeypatch.setenv("VGPU_GB_DIRECT_BITS", "6")
    if split:
        monkeypatch.setenv("VGPU_GB_SPLIT_ROWS", split)
    rng = np.random.default_rng(7)
    n = 200_000
    k = rng.integers(-3000, 3000, n).astype(np.int32)
    k[: n // 4] = 17  # one heavy key
    big = rng.integers(-(1 << 62), 1 << 62, n, dtype=np.int64)
    x = rng.standard_normal(n)
    plan = make_group_by(["k"], [make_aggregate(A.SUM, "v", T.HUGEINT), make_aggregate(A.MIN, "v", T.INT64),
                                 make_aggregate(A.MAX, "v", T.INT64), make_aggregate(A.SUM, "x", T.FLOAT64),
                                 make_aggregate(A.COUNT_STAR, "", T.INT64)],
                         make_scan(["k", "v", "x"]))
    r = GpuEngine.instance().execute_plan(plan, [make_column("k", T.INT32, k), make_column("v", T.INT64, big),
                                                 make_column("x", T.FLOAT64, x)])
    assert r.success, r.error_message
    keys = r.columns[0].data
    sums = hugeint_to_int(r.columns[1].data)
    order = np.argsort(k, kind="stable")
    uk, starts = np.unique(k[order], return_index=True)
    assert np.array_equal(np.sort(keys), uk)
    pos = {int(key): i for i, key in enumerate(keys.tolist())}
    bounds = list(starts) + [n]
    for j, key in enumerate(uk.tolist()):
        rows = order[bounds[j]:bounds[j + 1]]
        i = pos[key]
        assert sums[i] == int(big[rows].astype(object).sum())
        assert r.columns[2].data[i] == big[rows].min() and r.columns[3].data[i] == big[rows].max()
        assert r.columns[5].data[i] == len(rows)
        exp = float(np.sum(x[rows]))
        assert abs(r.columns[4].data[i] - exp) <= 1e-9 * max(1.0, float(np.sum(np.abs(x[rows]))))
