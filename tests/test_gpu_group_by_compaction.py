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
