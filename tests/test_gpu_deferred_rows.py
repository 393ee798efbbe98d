"""Device results executed without a sync (output_on_device, VGPU_EXEC_NO_SYNC): a root GROUP BY on the
one-pass path and a root FILTER/PROJECTION chain (over a scan or a cross product) leave their row count
on the device and the call returns without waiting; the count is read when the result's columns are
first asked for. Several such queries are queued before any is read, read back in another order, and
each equals the synchronous run of the same query and the oracle; a result freed unread and a global
aggregate (no keys: one row, read at once) behave."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from vectisdb_b200 import (ColumnCache, ExecuteOptions, GpuEngine, GpuTableRef, device_to_host, make_aggregate,
                           make_group_by, make_scan)
from vectisdb_b200 import workloads as W
from vectisdb_b200.engine import GpuAggregateKind as A, GpuValueType as T

pytestmark = pytest.mark.gpu


def _cached(wl):
    names = [c.name for c in wl.inputs]
    refs = []
    for table, cols in wl.tables.items():
        ref = GpuTableRef("memory", "main", table)
        ColumnCache.put_table(ref, [wl.inputs[names.index(c)] for c in cols])
        refs.append(ref)
    return refs


def _host(result, stream):
    return [device_to_host(c, stream) for c in result.columns]


def test_queued_no_sync_group_bys_read_their_counts_later():
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    wls = [W.c0(n=(1 << 20) + 37 * i, seed=20 + i, k_card=[1024, 700, 33, 1][i], table=f"defer_c0_{i}")
           for i in range(4)]
    refs = [r for wl in wls for r in _cached(wl)]
    eng = GpuEngine.instance()
    lazy = ExecuteOptions(serve_whole_scan_from_cache=True, output_on_device=True, no_sync=True, stream=sp)
    sync = ExecuteOptions(serve_whole_scan_from_cache=True, output_on_device=True, stream=sp)
    try:
        queued = [eng.execute_plan(wl.plan, [], lazy) for wl in wls for _ in range(2)]
        assert all(hasattr(r, "free") and r._columns is None for r in queued)
        for i in reversed(range(len(queued))):
            wl = wls[i // 2]
            got = _host(queued[i], sp)
            ref = eng.execute_plan(wl.plan, [], sync)
            want = _host(ref, sp)
            ref.free()
            assert [len(g) for g in got] == [len(w) for w in want]
            for g, w in zip(got, want):
                assert np.array_equal(g, w) or np.allclose(g, w, rtol=1e-12, atol=0)
            exp = O.c0(*[c.data for c in wl.inputs], wl.params["v_lt"], wl.params["w_mod"])
            assert np.array_equal(got[0], exp["k"]) and np.array_equal(got[2], exp["count"])
            assert np.array_equal(got[3], exp["min"]) and np.array_equal(got[4], exp["max"])
            assert np.allclose(got[1], exp["sum"], rtol=1e-12, atol=0)
            queued[i].free()
        # a result freed before anyone read it
        eng.execute_plan(wls[0].plan, [], lazy).free()
        torch.cuda.synchronize()
    finally:
        for ref in refs:
            ColumnCache.invalidate_table(ref)


def test_queued_no_sync_filters_read_their_counts_later():
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    cps = [W.cp(n=(1 << 20) + 11 * i, seed=30 + i, table=f"defer_cp_{i}") for i in range(2)]
    x = W.c2b(side=1000, seed=31)
    refs = [r for wl in cps + [x] for r in _cached(wl)]
    eng = GpuEngine.instance()
    lazy = ExecuteOptions(serve_whole_scan_from_cache=True, output_on_device=True, no_sync=True, stream=sp)
    try:
        queued = [eng.execute_plan(wl.plan, [], lazy) for wl in cps + [x, x]]
        assert all(r._columns is None for r in queued)
        for i in reversed(range(len(queued))):
            got = _host(queued[i], sp)
            queued[i].free()
            if i < len(cps):
                exp = O.cp(*[c.data for c in cps[i].inputs])
                assert len(got[0]) == len(exp["k"]) > 0
                assert np.array_equal(got[0], exp["k"]) and np.array_equal(got[2], exp["w"])
                assert np.array_equal(got[1], exp["v"])
            else:
                total, oa, ob = O.c2b(x.inputs[0].data, x.inputs[1].data, x.params["modulus"])
                assert len(got[0]) == total > 0
                assert np.array_equal(got[0], oa) and np.array_equal(got[1], ob)
    finally:
        for ref in refs:
            ColumnCache.invalidate_table(ref)


def test_no_sync_global_aggregate_has_its_one_row():
    stream = torch.cuda.Stream()
    wl = W.c0(n=1 << 16, seed=5, table="defer_global")
    refs = _cached(wl)
    try:
        plan = make_group_by([], [make_aggregate(A.COUNT_STAR, "", T.INT64), make_aggregate(A.SUM, "w", T.HUGEINT)],
                             make_scan(["k", "v", "w"], GpuTableRef("memory", "main", "defer_global")))
        r = GpuEngine.instance().execute_plan(plan, [], ExecuteOptions(serve_whole_scan_from_cache=True,
                                                                       output_on_device=True, no_sync=True,
                                                                       stream=stream.cuda_stream))
        got = _host(r, stream.cuda_stream)
        r.free()
        assert len(got[0]) == 1 and int(got[0][0]) == 1 << 16
    finally:
        for ref in refs:
            ColumnCache.invalidate_table(ref)
