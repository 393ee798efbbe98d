"""Device column cache semantics on the B200 (the reference's GpuColumnCache contract,
cuda_engine/src/gpu_column_cache.cpp:61-363):

- staging one column of a table again keeps the table's other committed columns resident (the
  reference keeps them so that hot column subsets stay cached, gpu_column_cache.cpp:163-172), the
  re-staged column takes its new contents, and invalidating the table drops every column;
- buffers read by a query that returned before its kernels finished (device output, no sync) are
  freed only after those kernels: the query's join table and cached columns are evicted while the
  query is still running and their memory is handed to a new table at once, and the result is still
  the one computed from the old contents.
"""
import numpy as np
import pytest

from vectisdb_b200 import (ColumnCache, ExecuteOptions, GpuEngine, GpuTableRef, device_to_host, make_aggregate,
                           make_column, make_group_by, make_join, make_scan)
from vectisdb_b200.engine import GpuAggregateKind as A, GpuValueType as T, hugeint_to_int

pytestmark = pytest.mark.gpu


def _scan_values(table, names, dtypes):
    r = GpuEngine.instance().execute_plan(make_scan(names, table), [], ExecuteOptions(serve_whole_scan_from_cache=True))
    assert r.success, r.error_message
    return [np.asarray(c.data).astype(d) for c, d in zip(r.columns, dtypes)]


def test_restaging_one_column_keeps_the_others():
    t = GpuTableRef("memory", "main", "keep_cols")
    rng = np.random.default_rng(3)
    n = 100_003
    a = rng.integers(-1000, 1000, n).astype(np.int64)
    b = rng.random(n)
    b2 = rng.random(n) + 5.0
    try:
        ColumnCache.put_table(t, [make_column("a", T.INT64, a), make_column("b", T.FLOAT64, b)])
        gen = ColumnCache.table_generation(t)
        before = ColumnCache.current_bytes()
        ColumnCache.begin_staging(t)
        assert ColumnCache.stage_chunk(t, make_column("b", T.FLOAT64, b2))
        ColumnCache.commit_staging(t, n)
        assert ColumnCache.table_generation(t) > gen
        assert ColumnCache.current_bytes() == before  # b replaced, a kept: same bytes resident
        got_a, got_b = _scan_values(t, ["a", "b"], [np.int64, np.float64])
        assert np.array_equal(got_a, a)
        assert np.array_equal(got_b, b2)
        assert ColumnCache.replayable_chunk_rows(t, ["a", "b"]) == [n]
        ColumnCache.invalidate_table(t)
        with pytest.raises(KeyError):
            ColumnCache.device_column(t, "a")
        with pytest.raises(KeyError):
            ColumnCache.device_column(t, "b")
    finally:
        ColumnCache.invalidate_table(t)


def test_eviction_while_a_no_sync_query_runs_waits_for_its_kernels():
    import torch
    rng = np.random.default_rng(21)
    nb, npr = 1 << 20, 1 << 24
    rk = rng.permutation(nb).astype(np.int64)
    rg = rng.integers(0, 512, nb).astype(np.int32)
    lk = rng.integers(0, nb + (nb >> 3), npr).astype(np.int64)  # about 1/9 of the probe rows miss
    lv = rng.integers(-1000, 1000, npr).astype(np.int64)
    t_b, t_p = GpuTableRef("memory", "main", "ev_build"), GpuTableRef("memory", "main", "ev_probe")
    t_n = GpuTableRef("memory", "main", "ev_new")
    plan = make_group_by(["rg"], [make_aggregate(A.SUM, "lv", T.HUGEINT), make_aggregate(A.COUNT_STAR, "", T.INT64)],
                         make_join("lk", "rk", ["rg", "lv"], make_scan(["lk", "lv"], t_p), make_scan(["rk", "rg"], t_b)))
    # expected: per rg, SUM(lv) and COUNT over matching probe rows
    pos = np.full(nb + (nb >> 3), -1, np.int64)
    pos[rk] = np.arange(nb)
    hit = pos[lk] >= 0
    g = rg[pos[lk[hit]]]
    exp_cnt = np.bincount(g, minlength=512)
    exp_sum = np.zeros(512, np.int64)
    np.add.at(exp_sum, g, lv[hit])
    stream = torch.cuda.Stream()
    opts = ExecuteOptions(serve_whole_scan_from_cache=True, output_on_device=True, no_sync=True,
                          stream=stream.cuda_stream)
    try:
        for trial in range(3):
            ColumnCache.put_table(t_p, [make_column("lk", T.INT64, lk), make_column("lv", T.INT64, lv)])
            ColumnCache.put_table(t_b, [make_column("rk", T.INT64, rk), make_column("rg", T.INT32, rg)])
            warm = GpuEngine.instance().execute_plan(plan, [], ExecuteOptions(serve_whole_scan_from_cache=True))
            assert warm.success, warm.error_message  # builds and keeps the join table
            r = GpuEngine.instance().execute_plan(plan, [], opts)  # returns before its kernels finish
            assert hasattr(r, "free"), r.error_message
            # evict everything it reads, then hand the memory to a new table of the same sizes at once
            ColumnCache.invalidate_table(t_b)
            ColumnCache.invalidate_table(t_p)
            junk = rng.integers(-(1 << 62), 1 << 62, npr).astype(np.int64)
            ColumnCache.put_table(t_n, [make_column("x", T.INT64, junk), make_column("y", T.INT64, junk[::-1].copy()),
                                        make_column("z", T.INT64, junk[:nb].copy()),
                                        make_column("w", T.INT32, junk[:nb].astype(np.int32))])
            keys = device_to_host(r.columns[0], stream.cuda_stream)
            sums = hugeint_to_int(device_to_host(r.columns[1], stream.cuda_stream))
            cnts = device_to_host(r.columns[2], stream.cuda_stream)
            r.free()
            got = {int(k): (int(s), int(c)) for k, s, c in zip(keys, sums, cnts)}
            assert got == {k: (int(exp_sum[k]), int(exp_cnt[k])) for k in range(512) if exp_cnt[k]}, trial
            ColumnCache.invalidate_table(t_n)
    finally:
        for t in (t_b, t_p, t_n):
            ColumnCache.invalidate_table(t)
