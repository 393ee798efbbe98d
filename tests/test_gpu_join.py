"""Equi-join under a pipeline: the fused forms (dense key tables holding a row index or the value
itself; sorted keys with a radix directory), with no materialized match pairs, against the
materializing form and against numpy, including misses, negative keys, keys below the right side's
minimum, and many-to-many fallback."""
import numpy as np
import pytest

from vectisdb_b200 import GpuEngine, make_aggregate, make_column, make_expr, make_filter, make_group_by, make_join, make_scan
from vectisdb_b200 import workloads as W
from vectisdb_b200.engine import GpuAggregateKind as A, GpuValueType as T
from oracle import oracle as O

pytestmark = pytest.mark.gpu
REL = 1e-12


def _close(got, exp):
    got, exp = np.asarray(got, np.float64), np.asarray(exp, np.float64)
    return np.all(np.abs(got - exp) <= REL * np.maximum(np.abs(exp), 1e-300))


def _run(plan, inputs):
    r = GpuEngine.instance().execute_plan(plan, inputs)
    assert r.success, r.error_message
    return r.columns


@pytest.mark.parametrize("fused", ["1", "0"])
def test_c2_join_group_by_fused_and_materialized(fused, monkeypatch):
    monkeypatch.setenv("VGPU_JOIN_FUSED", fused)
    wl = W.c2(probe_n=1 << 20, build_n=1 << 16, miss_lo=1 << 16, miss_span=1 << 16)
    pkey, x, bkey, g = [c.data for c in wl.inputs]
    gg, gs = [c.data for c in _run(wl.plan, wl.inputs)]
    order = np.argsort(gg)
    exp = O.c2(bkey, g, pkey, x)
    assert np.array_equal(gg[order], exp["g"])
    assert _close(gs[order], exp["sum"])


def _join_group_plan(key_type):
    left = make_scan(["lk", "lv"])
    right = make_scan(["rk", "rg"])
    join = make_join("lk", "rk", ["rg", "lv"], left, right)
    return make_group_by(["rg"], [make_aggregate(A.SUM, "lv", T.HUGEINT), make_aggregate(A.COUNT_STAR, "", T.INT64)],
                         join)


def _expected_join_group(lk, lv, rk, rg):
    import collections
    by_key = collections.defaultdict(list)
    for k, g in zip(rk.tolist(), rg.tolist()):
        by_key[k].append(g)
    sums, counts = collections.Counter(), collections.Counter()
    for k, v in zip(lk.tolist(), lv.tolist()):
        for g in by_key.get(k, ()):
            sums[g] += v
            counts[g] += 1
    return sums, counts


@pytest.mark.parametrize("dup", [False, True])
def test_join_group_with_negative_keys_misses_and_duplicates(dup):
    rng = np.random.default_rng(5)
    rk = rng.permutation(np.arange(-5000, 5000, dtype=np.int64))[:6000]
    if dup:
        rk[:500] = rk[500:1000]  # repeated right keys: the many-to-many path
    rg = rng.integers(0, 50, len(rk)).astype(np.int32)
    lk = rng.integers(-7000, 7000, 40000).astype(np.int64)  # misses on both sides of the key range
    lv = rng.integers(-1000, 1000, len(lk)).astype(np.int64)
    cols = _run(_join_group_plan(T.INT64), [make_column("lk", T.INT64, lk), make_column("lv", T.INT64, lv),
                                            make_column("rk", T.INT64, rk), make_column("rg", T.INT32, rg)])
    from vectisdb_b200.engine import hugeint_to_int
    got_g = cols[0].data.tolist()
    got_s = hugeint_to_int(cols[1].data)
    got_c = cols[2].data.tolist()
    sums, counts = _expected_join_group(lk, lv, rk, rg)
    assert sorted(got_g) == sorted(counts)
    for g, s, c in zip(got_g, got_s, got_c):
        assert s == sums[g] and c == counts[g]


def test_filter_over_fused_join_keeps_left_order():
    rng = np.random.default_rng(9)
    rk = rng.permutation(np.arange(1000, 3000, dtype=np.int32))
    rv = rng.integers(0, 100, len(rk)).astype(np.int32)
    lk = rng.integers(0, 4000, 30000).astype(np.int32)
    lv = np.arange(len(lk), dtype=np.int64)
    join = make_join("lk", "rk", ["lv", "rv"], make_scan(["lk", "lv"]), make_scan(["rk", "rv"]))
    plan = make_filter([make_expr("((bool*)out)[idx] = (((const int*)inputs[0])[row] % 3) == 0;", ["rv"],
                                  T.BOOLEAN)], join)
    cols = _run(plan, [make_column("lk", T.INT32, lk), make_column("lv", T.INT64, lv), make_column("rk", T.INT32, rk),
                       make_column("rv", T.INT32, rv)])
    pos = {int(k): i for i, k in enumerate(rk.tolist())}
    exp_lv, exp_rv = [], []
    for k, v in zip(lk.tolist(), lv.tolist()):
        i = pos.get(k)
        if i is not None and rv[i] % 3 == 0:
            exp_lv.append(v)
            exp_rv.append(int(rv[i]))
    assert np.array_equal(cols[0].data, np.array(exp_lv, np.int64))  # left-major order
    assert np.array_equal(cols[1].data, np.array(exp_rv, np.int32))


@pytest.mark.parametrize("layout", ["dense_rows", "sorted_directory"])
def test_fused_join_table_forms_match_numpy(layout):
    """Dense keys with two right columns (row-index table) and sparse keys (sorted keys + radix
    directory): every left row finds its right row or none, left order kept."""
    rng = np.random.default_rng(21)
    if layout == "dense_rows":
        rk = rng.permutation(np.arange(-3000, 3000, dtype=np.int64))
    else:
        rk = np.unique(rng.integers(-(1 << 40), 1 << 40, 5000)).astype(np.int64)
        rng.shuffle(rk)
    r1 = rng.integers(0, 1000, len(rk)).astype(np.int32)
    r2 = rng.standard_normal(len(rk))
    lk = np.concatenate([rng.choice(rk, 20000), rng.integers(-(1 << 41), 1 << 41, 5000)]).astype(np.int64)
    rng.shuffle(lk)
    lv = np.arange(len(lk), dtype=np.int64)
    join = make_join("lk", "rk", ["lv", "r1", "r2"], make_scan(["lk", "lv"]), make_scan(["rk", "r1", "r2"]))
    plan = make_filter([make_expr("((bool*)out)[idx] = ((const int*)inputs[0])[row] >= 0;", ["r1"], T.BOOLEAN)], join)
    cols = _run(plan, [make_column("lk", T.INT64, lk), make_column("lv", T.INT64, lv), make_column("rk", T.INT64, rk),
                       make_column("r1", T.INT32, r1), make_column("r2", T.FLOAT64, r2)])
    pos = {int(k): i for i, k in enumerate(rk.tolist())}
    exp = [(v, pos[k]) for k, v in zip(lk.tolist(), lv.tolist()) if k in pos]
    assert np.array_equal(cols[0].data, np.array([v for v, _ in exp], np.int64))
    assert np.array_equal(cols[1].data, r1[[i for _, i in exp]])
    assert np.array_equal(cols[2].data, r2[[i for _, i in exp]])


@pytest.mark.parametrize("values,vtype", [
    ("small", T.INT32),      # offsets below 255: 1-byte table
    ("medium", T.INT32),     # below 65535: 2-byte table
    ("wide", T.INT32),       # 4-byte table with the all-ones marker
    ("full", T.INT32),       # -1 and 0 together span every 32-bit pattern: the 8-byte table stays
    ("negative", T.INT32),   # all negative, a narrow span of high bit patterns
    ("short", T.INT16),      # a 2-byte right column, negative values included
])
def test_dense_inline_table_widths(values, vtype, monkeypatch):
    """The single right column inlined into the dense key table, narrowed to the fewest bytes that hold
    every value's offset from the smallest: the same matches and values as numpy and as the 8-byte form."""
    rng = np.random.default_rng(31)
    rk = rng.permutation(np.arange(0, 50000, dtype=np.int64))
    n_r = len(rk)
    np_t = np.int16 if vtype == T.INT16 else np.int32
    rv = {"small": lambda: rng.integers(7, 200, n_r), "medium": lambda: rng.integers(-30000, 30000, n_r),
          "wide": lambda: rng.integers(-(1 << 30), 1 << 30, n_r),
          "full": lambda: np.where(rng.random(n_r) < 0.5, -1, rng.integers(0, 1 << 31, n_r)),
          "negative": lambda: rng.integers(-90, -1, n_r), "short": lambda: rng.integers(-32768, 32767, n_r)}[values]()
    rv = rv.astype(np_t)
    lk = rng.integers(-1000, 60000, 200000).astype(np.int64)
    lv = np.arange(len(lk), dtype=np.int64)
    join = make_join("lk", "rk", ["lv", "rv"], make_scan(["lk", "lv"]), make_scan(["rk", "rv"]))
    plan = make_filter([make_expr("((bool*)out)[idx] = ((const long long*)inputs[0])[row] % 2 == 0;", ["lv"],
                                  T.BOOLEAN)], join)
    inputs = [make_column("lk", T.INT64, lk), make_column("lv", T.INT64, lv), make_column("rk", T.INT64, rk),
              make_column("rv", vtype, rv)]
    pos = np.full(60000, -1, np.int64)
    pos[rk] = np.arange(n_r)
    hit = (lk >= 0) & (lk < 60000)
    hit[hit] = pos[lk[hit]] >= 0
    keep = hit & (lv % 2 == 0)
    exp_rv = rv[pos[lk[keep]]]
    res = {}
    for compact in ("1", "0"):
        monkeypatch.setenv("VGPU_JOIN_COMPACT", compact)
        cols = _run(plan, inputs)
        assert np.array_equal(cols[0].data, lv[keep])
        assert np.array_equal(cols[1].data, exp_rv)
        res[compact] = cols[1].data
    assert np.array_equal(res["1"], res["0"])


def test_join_table_kept_across_queries_until_invalidated():
    """A right side read from the column cache: the second identical join reuses the dense table built
    by the first (no build launch), and after the build table is invalidated and staged again with new
    payload values the join rebuilds and returns the new values."""
    from vectisdb_b200 import ColumnCache, ExecuteOptions, GpuTableRef
    from vectisdb_b200.engine import profile_drain, profile_enable
    rng = np.random.default_rng(17)
    rk = rng.permutation(np.arange(0, 40000, dtype=np.int64))
    lk = rng.integers(-100, 45000, 150000).astype(np.int64)
    lv = rng.integers(-1000, 1000, len(lk)).astype(np.int64)
    t_b, t_p = GpuTableRef("memory", "main", "jc_build"), GpuTableRef("memory", "main", "jc_probe")
    ColumnCache.put_table(t_p, [make_column("lk", T.INT64, lk), make_column("lv", T.INT64, lv)])
    plan = make_group_by(["rg"], [make_aggregate(A.SUM, "lv", T.HUGEINT), make_aggregate(A.COUNT_STAR, "", T.INT64)],
                         make_join("lk", "rk", ["rg", "lv"], make_scan(["lk", "lv"], t_p), make_scan(["rk", "rg"], t_b)))
    opts = ExecuteOptions(serve_whole_scan_from_cache=True)
    from vectisdb_b200.engine import hugeint_to_int

    def run(rg):
        profile_enable(True)
        profile_drain()
        try:
            r = GpuEngine.instance().execute_plan(plan, [], opts)
            names = [k for k, _, _, _ in profile_drain()]
        finally:
            profile_enable(False)
        assert r.success, r.error_message
        sums, counts = _expected_join_group(lk, lv, rk, rg)
        got = dict(zip(r.columns[0].data.tolist(), zip(hugeint_to_int(r.columns[1].data), r.columns[2].data.tolist())))
        assert got == {g: (sums[g], counts[g]) for g in counts}
        return names

    try:
        rg1 = rng.integers(0, 300, len(rk)).astype(np.int32)
        ColumnCache.put_table(t_b, [make_column("rk", T.INT64, rk), make_column("rg", T.INT32, rg1)])
        assert "join_dense_table" in run(rg1)
        assert "join_dense_table" not in run(rg1)  # kept
        ColumnCache.invalidate_table(t_b)
        rg2 = rng.integers(1000, 1200, len(rk)).astype(np.int32)
        ColumnCache.put_table(t_b, [make_column("rk", T.INT64, rk), make_column("rg", T.INT32, rg2)])
        assert "join_dense_table" in run(rg2)  # new contents: rebuilt
        assert "join_dense_table" not in run(rg2)
    finally:
        ColumnCache.invalidate_table(t_b)
        ColumnCache.invalidate_table(t_p)


def _launched(fn):
    from vectisdb_b200.engine import profile_drain, profile_enable
    profile_enable(True)
    profile_drain()
    try:
        out = fn()
        names = [k for k, _, _, _ in profile_drain()]
    finally:
        profile_enable(False)
    return out, names


def test_repeated_build_keys_fuse_into_the_group_by():
    """The join + group-by with every build key repeated (the c2 shape with two build rows per key):
    each probe row expands into its matches inside the group-by kernel -- no match pairs are
    materialized -- read from the dense multi-match table (two 12-bit slots per 4-byte entry, filled
    without sorting), and the result equals the oracle's hash join."""
    wl = W.c2dup(probe_n=1 << 22, build_n=1 << 20)
    pkey, x, bkey, g = [c.data for c in wl.inputs]
    (gg, gs), names = _launched(lambda: [c.data for c in _run(wl.plan, wl.inputs)])
    assert "join_dense_multi" in names and "radix_scatter" not in names, names
    assert "join_runs" not in names and "join_expand" not in names, names
    exp = O.c2(bkey, g, pkey, x)
    order = np.argsort(gg)
    assert np.array_equal(gg[order], exp["g"])
    assert _close(gs[order], exp["sum"])


@pytest.mark.parametrize("repeat,card,path", [
    (2, 1 << 20, "wide"),     # 20-bit values: one 4-byte entry holds one slot, an 8-byte one three
    (5, 4096, "wide"),        # five 12-bit slots need the 8-byte entry
    (6, 4096, "sorted"),      # more matches than an entry holds: the sorted runs
    (3, 2, "narrow"),         # 1-bit values, three slots in 4 bytes
])
def test_join_group_by_over_repeated_keys_every_table_form(repeat, card, path):
    """A join + group-by whose right keys each repeat `repeat` times, with right values of `card`
    distinct values: the dense multi-match table in 4- or 8-byte entries while the matches fit its
    slots, the sorted runs when a key has more; exact HUGEINT sums and counts per group against a
    Python hash join, misses and negative probe keys included (the dense forms index the right keys'
    zero-extended range, so the right keys here are non-negative)."""
    rng = np.random.default_rng(40 + repeat)
    base = rng.permutation(np.arange(0, 40_000, dtype=np.int64))[:30_000]
    rk = np.repeat(base, repeat)[rng.permutation(30_000 * repeat)]
    rg = rng.integers(0, card, len(rk)).astype(np.int32)
    lk = rng.integers(-5_000, 45_000, 400_000).astype(np.int64)
    lv = rng.integers(-(1 << 40), 1 << 40, len(lk)).astype(np.int64)
    cols, names = _launched(lambda: _run(_join_group_plan(T.INT64), [
        make_column("lk", T.INT64, lk), make_column("lv", T.INT64, lv),
        make_column("rk", T.INT64, rk), make_column("rg", T.INT32, rg)]))
    if path == "sorted":
        assert "radix_scatter" in names and "join_expand" not in names, names
    else:
        assert "join_dense_multi" in names and "radix_scatter" not in names, names
    from vectisdb_b200.engine import hugeint_to_int
    sums, counts = _expected_join_group(lk, lv, rk, rg)
    got = dict(zip(cols[0].data.tolist(), zip(hugeint_to_int(cols[1].data), cols[2].data.tolist())))
    assert got == {k: (sums[k], counts[k]) for k in counts}


@pytest.mark.parametrize("repeat", [2, 7])
def test_filter_over_multi_match_join_keeps_left_then_right_order(repeat):
    """A filter over a join whose right keys repeat: outputs are left-major, and a left row's matches
    follow the right side's original order (the stable sort), as the reference's join emits them."""
    rng = np.random.default_rng(31 + repeat)
    base = rng.permutation(np.arange(-3000, 3000, dtype=np.int64))[:2500]
    rk = np.concatenate([base] * repeat)[rng.permutation(2500 * repeat)]
    rv = rng.integers(0, 1000, len(rk)).astype(np.int32)
    lk = rng.integers(-4000, 4000, 50000).astype(np.int64)
    lv = np.arange(len(lk), dtype=np.int64)
    join = make_join("lk", "rk", ["lv", "rv"], make_scan(["lk", "lv"]), make_scan(["rk", "rv"]))
    plan = make_filter([make_expr("((bool*)out)[idx] = (((const int*)inputs[0])[row] % 3) != 1;", ["rv"],
                                  T.BOOLEAN)], join)
    cols, names = _launched(lambda: _run(plan, [make_column("lk", T.INT64, lk), make_column("lv", T.INT64, lv),
                                                make_column("rk", T.INT64, rk), make_column("rv", T.INT32, rv)]))
    assert "join_expand" not in names, names
    by_key = {}
    for i, k in enumerate(rk.tolist()):
        by_key.setdefault(k, []).append(i)
    exp_lv, exp_rv = [], []
    for k, v in zip(lk.tolist(), lv.tolist()):
        for i in by_key.get(k, ()):
            if rv[i] % 3 != 1:
                exp_lv.append(v)
                exp_rv.append(int(rv[i]))
    assert np.array_equal(cols[0].data, np.array(exp_lv, np.int64))
    assert np.array_equal(cols[1].data, np.array(exp_rv, np.int32))


def test_multi_match_join_under_a_high_cardinality_group_by():
    """Grouping a repeated-key join by a key with too many values for the one-pass tables: the matches
    are expanded into a relation first, then partitioned; exact sums and counts."""
    rng = np.random.default_rng(12)
    rk = np.repeat(rng.permutation(200_000).astype(np.int64), 3)
    rg = rng.integers(0, 1 << 20, len(rk)).astype(np.int32)
    lk = rng.integers(0, 220_000, 300_000).astype(np.int64)
    lv = rng.integers(-1000, 1000, len(lk)).astype(np.int64)
    cols = _run(_join_group_plan(T.INT64), [make_column("lk", T.INT64, lk), make_column("lv", T.INT64, lv),
                                            make_column("rk", T.INT64, rk), make_column("rg", T.INT32, rg)])
    from vectisdb_b200.engine import hugeint_to_int
    sums, counts = _expected_join_group(lk, lv, rk, rg)
    got = dict(zip(cols[0].data.tolist(), zip(hugeint_to_int(cols[1].data), cols[2].data.tolist())))
    assert got == {g: (sums[g], counts[g]) for g in counts}


def test_very_long_runs_use_the_load_balanced_join():
    """A right key repeated more than 65536 times is spread over many threads by the materializing
    join's expansion instead of one thread walking the run."""
    rk = np.concatenate([np.full(70_000, 5, np.int64), np.arange(10, 1010, dtype=np.int64)])
    rg = (np.arange(len(rk)) % 17).astype(np.int32)
    lk = np.array([5, 6, 10, 5, 1009, 2000], np.int64)
    lv = np.array([1, 2, 3, 4, 5, 6], np.int64)
    cols, names = _launched(lambda: _run(_join_group_plan(T.INT64), [make_column("lk", T.INT64, lk),
                                                                      make_column("lv", T.INT64, lv),
                                                                      make_column("rk", T.INT64, rk),
                                                                      make_column("rg", T.INT32, rg)]))
    assert "join_expand" in names, names
    from vectisdb_b200.engine import hugeint_to_int
    sums, counts = _expected_join_group(lk, lv, rk, rg)
    got = dict(zip(cols[0].data.tolist(), zip(hugeint_to_int(cols[1].data), cols[2].data.tolist())))
    assert got == {g: (sums[g], counts[g]) for g in counts}

