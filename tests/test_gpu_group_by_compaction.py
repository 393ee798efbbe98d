"""The one-pass group-by's two compaction forms on the B200: in the CTA that finishes its merge last
(behind a ticket), and -- when the ticket's argument word would reach the reserved key words -- in a
separate single-CTA final kernel. GROUP BY k with MIN over 21 (fused) and 22 (separate) INT64 columns
against numpy, with a negative key range, keys with no rows, and several launches' worth of rows."""
import numpy as np
import pytest

from vectisdb_b200 import GpuEngine, make_aggregate, make_column, make_group_by, make_scan
from vectisdb_b200.engine import GpuAggregateKind as A, GpuTableRef, GpuValueType as T, profile_drain, profile_enable

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,fused", [(21, True), (22, False)])
def test_min_per_column_group_by_in_both_compaction_forms(m, fused):
    rng = np.random.default_rng(60 + m)
    n = 300_001
    k = rng.integers(-300, 212, n).astype(np.int32)  # 512 key slots: the tables fit the one-pass bound
    k[k == 5] = 6  # a key value inside the range with no rows
    xs = [rng.integers(-(1 << 62), 1 << 62, n).astype(np.int64) for _ in range(m)]
    cols = [make_column("k", T.INT32, k)] + [make_column(f"x{i}", T.INT64, x) for i, x in enumerate(xs)]
    plan = make_group_by(["k"], [make_aggregate(A.MIN, f"x{i}", T.INT64) for i in range(m)],
                         make_scan([c.name for c in cols], GpuTableRef("memory", "main", f"minw{m}")))
    profile_drain()
    profile_enable(True)
    try:
        r = GpuEngine.instance().execute_plan(plan, cols)
        names = [rec[0] for rec in profile_drain()]
    finally:
        profile_enable(False)
    assert r.success, r.error_message
    assert ("vgpu_gb_direct_final" in names) == (not fused), names
    keys = np.unique(k)
    order = np.argsort(k, kind="stable")
    starts = np.searchsorted(k[order], keys)
    assert np.array_equal(np.asarray(r.columns[0].data), keys)
    for i, x in enumerate(xs):
        assert np.array_equal(np.asarray(r.columns[1 + i].data), np.minimum.reduceat(x[order], starts)), i


def test_min_max_over_cached_integer_columns_with_32_bit_offsets():
    """MIN/MAX over cached integer columns whose values span less than 2^32 keep 32-bit offsets from the
    column minimum in the one-pass kernel's shared tables: INT32 over its whole range (offsets up to
    2^32 - 1), INT64 around zero just inside the bound, INT16 -- and an INT64 column spanning more than
    2^32 keeps 64-bit state. Every result equals numpy's."""
    from vectisdb_b200 import ColumnCache
    rng = np.random.default_rng(77)
    n = 400_003
    k = rng.integers(0, 1000, n).astype(np.int32)
    i32 = rng.integers(-(1 << 31), 1 << 31, n, dtype=np.int64).astype(np.int32)
    i32[:2] = [-(1 << 31), (1 << 31) - 1]
    i64 = rng.integers(-(1 << 31) + 5, (1 << 31) + 4, n).astype(np.int64)
    wide = rng.integers(-(1 << 40), 1 << 40, n).astype(np.int64)
    i16 = rng.integers(-(1 << 15), 1 << 15, n).astype(np.int16)
    cols = [make_column("k", T.INT32, k), make_column("a", T.INT32, i32), make_column("b", T.INT64, i64),
            make_column("c", T.INT64, wide), make_column("d", T.INT16, i16)]
    ref = GpuTableRef("memory", "main", "minmax32")
    ColumnCache.put_table(ref, cols)
    try:
        aggs = []
        for name, out in (("a", T.INT32), ("b", T.INT64), ("c", T.INT64), ("d", T.INT16)):
            aggs += [make_aggregate(A.MIN, name, out), make_aggregate(A.MAX, name, out)]
        plan = make_group_by(["k"], aggs, make_scan(["k", "a", "b", "c", "d"], ref))
        from vectisdb_b200 import ExecuteOptions
        r = GpuEngine.instance().execute_plan(plan, [], ExecuteOptions(serve_whole_scan_from_cache=True))
        assert r.success, r.error_message
        keys = np.unique(k)
        order = np.argsort(k, kind="stable")
        starts = np.searchsorted(k[order], keys)
        assert np.array_equal(np.asarray(r.columns[0].data), keys)
        for j, x in enumerate((i32, i64, wide, i16)):
            xs = x[order]
            assert np.array_equal(np.asarray(r.columns[1 + 2 * j].data), np.minimum.reduceat(xs, starts)), j
            assert np.array_equal(np.asarray(r.columns[2 + 2 * j].data), np.maximum.reduceat(xs, starts)), j
    finally:
        ColumnCache.invalidate_table(ref)
