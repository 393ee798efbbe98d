"""Heavy-key pre-aggregation of the direct-partitioned group-by: rows of the most frequent keys are
folded into per-CTA partial states during the scatter and reach the bucket pass as one partial
record per key and CTA. Results must be the ones without it, bit-exact for integer, DECIMAL and COUNT
aggregates and within 1e-12 relative for DOUBLE sums: on skewed and on uniform keys, with split
partitions, with partial sums that leave 64 bits (the query then reruns without pre-aggregation)."""
import numpy as np
import pytest

from vectisdb_b200 import GpuEngine, make_aggregate, make_column, make_group_by, make_scan
from vectisdb_b200 import workloads as W
from vectisdb_b200.engine import GpuAggregateKind as A, GpuValueType as T, hugeint_to_int, profile_drain, profile_enable
from oracle import oracle as O

pytestmark = pytest.mark.gpu
REL = 1e-12


def _close(got, exp):
    got, exp = np.asarray(got, np.float64), np.asarray(exp, np.float64)
    return np.all(np.abs(got - exp) <= REL * np.maximum(np.abs(exp), 1e-300))


def _launched(fn):
    profile_enable(True)
    profile_drain()
    try:
        out = fn()
        names = [k for k, _, _, _ in profile_drain()]
    finally:
        profile_enable(False)
    return out, names


def _check_c1(wl, cols):
    a, b, amt, v, ts = [c.data for c in wl.inputs]
    ga, gb, gsum, gavg, gcnt, gmax = [c.data for c in cols]
    order = np.lexsort((gb, ga))
    exp = O.c1(a, b, amt, v, ts, wl.params["ts_gt"])
    assert len(ga) == len(exp["a"])
    assert np.array_equal(ga[order], exp["a"]) and np.array_equal(gb[order], exp["b"])
    assert np.array_equal(gcnt[order], exp["count"]) and np.array_equal(gmax[order], exp["max"])
    gs = gsum[order]
    assert np.array_equal(gs["lower"], exp["sum_lo"]) and np.array_equal(gs["upper"], exp["sum_hi"])
    assert _close(gavg[order], exp["avg"])


@pytest.mark.parametrize("n,env", [
    (1 << 14, {}),                                          # a handful of CTAs, every sampled key heavy
    (1 << 18, {}),
    (1 << 18, {"VGPU_GB_SPLIT_ROWS": "256"}),               # split partitions merged through global tables
    (1 << 18, {"VGPU_GB_DIRECT_BITS": "8", "VGPU_GB_BUCKET_THREADS": "128"}),
    (1 << 18, {"VGPU_GB_HEAVY_KEYS": "8"}),                 # few keys: the threshold caps the selection
    ((1 << 20) + 12345, {}),                                # staged tiles with a partial tail tile
    ((1 << 20) + 12345, {"VGPU_GB_STAGED": "0"}),           # the same through per-thread loads
])
def test_c1_forced_heavy_keys_match_oracle(n, env, monkeypatch):
    monkeypatch.setenv("VGPU_GB_STRATEGY", "direct")
    monkeypatch.setenv("VGPU_GB_HEAVY", "2")
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    wl = W.c1(n=n)
    r, names = _launched(lambda: GpuEngine.instance().execute_plan(wl.plan, wl.inputs))
    assert r.success, r.error_message
    assert "vgpu_gb_sample" in names and "heavy_select" in names
    _check_c1(wl, r.columns)


def test_c1_heavy_keys_chosen_on_skewed_input():
    """Default settings at 2^22 rows of the Zipf(1.1) keys: the sample finds heavy keys by itself."""
    wl = W.c1(n=1 << 22)
    r, names = _launched(lambda: GpuEngine.instance().execute_plan(wl.plan, wl.inputs))
    assert r.success, r.error_message
    assert "vgpu_gb_sample" in names
    assert names.count("vgpu_gb_part_scatter") == 1
    _check_c1(wl, r.columns)


def _generic_plan(table=None):
    return make_group_by(["k"], [
        make_aggregate(A.SUM, "v", T.HUGEINT), make_aggregate(A.MIN, "w", T.INT64),
        make_aggregate(A.MAX, "u", T.INT64), make_aggregate(A.SUM, "x", T.FLOAT64),
        make_aggregate(A.AVG, "y", T.FLOAT64), make_aggregate(A.COUNT, "z", T.INT64),
        make_aggregate(A.COUNT_STAR, "", T.INT64)], make_scan(["k", "v", "w", "u", "x", "y", "z"], table))


@pytest.mark.parametrize("resident", [False, True])
@pytest.mark.parametrize("big", [False, True])
def test_heavy_partials_of_every_aggregate_kind(big, resident, monkeypatch):
    """SUM/MIN/MAX/AVG over BIGINT, SUM over DOUBLE, COUNT(col), COUNT(*) with one very heavy key and
    negative values. With values near 2^62 a CTA's partial sum leaves 64 bits: the launch is flagged
    and the query reruns without pre-aggregation, exact all the same. Also with the columns served from
    the column cache (ranges known, no host copy)."""
    monkeypatch.setenv("VGPU_GB_STRATEGY", "direct")
    monkeypatch.setenv("VGPU_GB_DIRECT_BITS", "6")
    monkeypatch.setenv("VGPU_GB_HEAVY", "2")
    rng = np.random.default_rng(11)
    n = 300_000
    k = rng.integers(-3000, 3000, n).astype(np.int32)
    k[rng.random(n) < 0.3] = 17
    k[rng.random(n) < 0.1] = -2999
    lim = 1 << 62 if big else 1 << 40
    v = rng.integers(-lim, lim, n, dtype=np.int64)
    if big:
        v[k == 17] = (1 << 62) - rng.integers(0, 1000, int((k == 17).sum()))
    w = rng.integers(-(1 << 50), 1 << 50, n, dtype=np.int64)
    u = rng.integers(-(1 << 50), 1 << 50, n, dtype=np.int64)
    x = rng.standard_normal(n)
    y = rng.integers(-1000, 1000, n, dtype=np.int64)
    z = rng.integers(0, 5, n, dtype=np.int64)
    cols = [make_column("k", T.INT32, k), make_column("v", T.INT64, v), make_column("w", T.INT64, w),
            make_column("u", T.INT64, u), make_column("x", T.FLOAT64, x), make_column("y", T.INT64, y),
            make_column("z", T.INT64, z)]
    if resident:
        from vectisdb_b200 import ColumnCache, ExecuteOptions, GpuTableRef
        ref = GpuTableRef("memory", "main", f"heavy_generic_{int(big)}")
        ColumnCache.put_table(ref, cols)
        try:
            r, names = _launched(lambda: GpuEngine.instance().execute_plan(
                _generic_plan(ref), [], ExecuteOptions(serve_whole_scan_from_cache=True)))
        finally:
            ColumnCache.invalidate_table(ref)
    else:
        r, names = _launched(lambda: GpuEngine.instance().execute_plan(_generic_plan(), cols))
    assert r.success, r.error_message
    assert "vgpu_gb_sample" in names
    if big:
        assert names.count("vgpu_gb_part_scatter") == 2  # flagged, rerun without pre-aggregation
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
        assert sums[i] == int(v[rows].astype(object).sum())
        assert r.columns[2].data[i] == w[rows].min() and r.columns[3].data[i] == u[rows].max()
        exp_x = float(np.sum(x[rows]))
        assert abs(r.columns[4].data[i] - exp_x) <= 1e-9 * max(1.0, float(np.sum(np.abs(x[rows]))))
        exp_avg = int(y[rows].astype(object).sum()) / len(rows)
        assert abs(r.columns[5].data[i] - exp_avg) <= REL * max(1.0, abs(exp_avg))
        assert r.columns[6].data[i] == len(rows) and r.columns[7].data[i] == len(rows)


def test_heavy_off_and_on_agree_on_uniform_keys(monkeypatch):
    """Uniform keys: forced pre-aggregation selects keys with a few sampled rows (one per partition at
    most), so most CTAs write partial records of keys they never saw (count 0, skipped by the bucket
    pass)."""
    monkeypatch.setenv("VGPU_GB_STRATEGY", "direct")
    rng = np.random.default_rng(3)
    n = 1 << 19
    a = rng.integers(0, 1 << 14, n).astype(np.int32)
    b = rng.integers(0, 4, n).astype(np.int32)
    amt = rng.integers(-(1 << 30), 1 << 30, n, dtype=np.int64)
    x = rng.random(n)
    plan = make_group_by(["a", "b"], [make_aggregate(A.SUM, "amt", T.HUGEINT), make_aggregate(A.SUM, "x", T.FLOAT64),
                                      make_aggregate(A.COUNT_STAR, "", T.INT64)], make_scan(["a", "b", "amt", "x"]))
    cols = [make_column("a", T.INT32, a), make_column("b", T.INT32, b), make_column("amt", T.INT64, amt),
            make_column("x", T.FLOAT64, x)]
    res = {}
    for mode in ("0", "2"):
        monkeypatch.setenv("VGPU_GB_HEAVY", mode)
        r = GpuEngine.instance().execute_plan(plan, cols)
        assert r.success, r.error_message
        ga, gb = r.columns[0].data, r.columns[1].data
        order = np.lexsort((gb, ga))
        res[mode] = [c.data[order] for c in r.columns]
    for c_off, c_on in zip(res["0"][:2], res["2"][:2]):
        assert np.array_equal(c_off, c_on)
    assert np.array_equal(res["0"][2], res["2"][2]) and np.array_equal(res["0"][4], res["2"][4])
    assert _close(res["2"][3], res["0"][3])
