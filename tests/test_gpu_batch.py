"""Batching: many C0-shaped filter + group-by queries in one persistent, graph-captured launch must
give each query the same groups and aggregates as running it alone (COUNT/MIN/MAX bit-exact, FP64
sums within 1e-12 relative) and as the oracle."""
import numpy as np
import pytest

from vectisdb_b200 import (BatchOptions, ColumnCache, ExecuteOptions, GpuEngine, GpuTableRef, batch_clear,
                           device_to_host)
from vectisdb_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

REL = 1e-12


def _close(got, exp):
    got = np.asarray(got, np.float64)
    exp = np.asarray(exp, np.float64)
    return np.all(np.abs(got - exp) <= REL * np.maximum(np.abs(exp), 1e-300))


def _check_against_oracle(wl, cols):
    k, s, c, mn, mx = [x.data for x in cols]
    order = np.argsort(k)
    exp = O.c0(wl.inputs[0].data, wl.inputs[1].data, wl.inputs[2].data, wl.params["v_lt"], wl.params["w_mod"])
    assert np.array_equal(k[order], exp["k"])
    assert np.array_equal(c[order], exp["count"])
    assert np.array_equal(mn[order], exp["min"]) and np.array_equal(mx[order], exp["max"])
    assert _close(s[order], exp["sum"])


def _small_batch(n=24, **kw):
    return W.c3(n_queries=n, min_log2=10, max_log2=16, card_lo=16, card_hi=4096, **kw)


@pytest.mark.parametrize("bopts", [BatchOptions(use_graph=False), BatchOptions(smem_slots=256, tile_rows=4096),
                                   BatchOptions(block=512, items=8, tile_rows=65536)])
def test_batch_matches_oracle_and_solo_runs(bopts):
    wls = _small_batch()
    eng = GpuEngine.instance()
    results, stats = eng.execute_batch([w.plan for w in wls], [w.inputs for w in wls], batch=bopts)
    assert stats["batched"] == len(wls) and stats["fallback"] == 0 and stats["templates"] == 1
    for wl, r in zip(wls, results):
        _check_against_oracle(wl, r.columns)
        solo = eng.execute_plan(wl.plan, wl.inputs)
        assert solo.success, solo.error_message
        a, b = r.columns, solo.columns
        oa, ob = np.argsort(a[0].data), np.argsort(b[0].data)
        for i in (0, 2, 3, 4):
            assert np.array_equal(a[i].data[oa], b[i].data[ob])
        assert _close(a[1].data[oa], b[1].data[ob])


def test_batch_graph_replay_from_cache_on_device():
    """Resident columns, device outputs, a torch stream: the second call replays the captured graph."""
    torch = pytest.importorskip("torch")
    batch_clear()
    wls = _small_batch(n=16)
    for w in wls:
        for table, names in w.tables.items():
            ColumnCache.put_table(GpuTableRef("memory", "main", table), w.inputs)
    eng = GpuEngine.instance()
    stream = torch.cuda.Stream()
    opts = ExecuteOptions(serve_whole_scan_from_cache=True, output_on_device=True, stream=stream.cuda_stream)
    first = None
    prepared = eng.prepare_batch([w.plan for w in wls])
    for call in range(3):
        # the first call passes the plans, the next ones the prepared batch: same template, same graph
        src = [w.plan for w in wls] if call == 0 else prepared
        results, stats = eng.execute_batch(src, [[] for _ in wls], opts)
        assert stats["batched"] == len(wls)
        if call > 0:
            assert stats["graph_replays"] == 1
        host = [[device_to_host(c, stream.cuda_stream) for c in r.columns] for r in results]
        for r in results:
            r.free()
        if first is None:
            first = host
        else:
            for a, b in zip(first, host):
                for i, (x, y) in enumerate(zip(a, b)):
                    # FP64 sums are order-dependent across runs: within the tolerance, the rest exact
                    assert _close(x, y) if i == 1 else np.array_equal(x, y)
    for wl, cols in zip(wls, first):
        class _C:
            def __init__(self, d):
                self.data = d
        _check_against_oracle(wl, [_C(x) for x in cols])
    for w in wls:
        for table in w.tables:
            ColumnCache.invalidate_table(GpuTableRef("memory", "main", table))


def test_batch_mixes_templates_and_falls_back():
    """Two templates (different filter shapes) in one call, plus a plan the batch form does not take:
    every result still matches its solo run."""
    eng = GpuEngine.instance()
    wls = _small_batch(n=6)
    other = W.c0(n=5000, seed=99, k_card=100, v_lt=0.3, w_mod=5)
    other.plan.children[0].children[0].expressions = other.plan.children[0].children[0].expressions[:1]
    cross = W.c2b(side=64)  # FILTER over CROSS_PRODUCT: outside the batch form
    plans = [w.plan for w in wls] + [other.plan, cross.plan]
    inputs = [w.inputs for w in wls] + [other.inputs, cross.inputs]
    results, stats = eng.execute_batch(plans, inputs)
    assert stats["templates"] == 2 and stats["batched"] == len(wls) + 1 and stats["fallback"] == 1
    for p, ins, r in zip(plans, inputs, results):
        solo = eng.execute_plan(p, ins)
        assert solo.success
        assert len(r.columns) == len(solo.columns)
        assert r.columns[0].row_count == solo.columns[0].row_count


def test_batch_autotune_picks_a_geometry_and_stays_exact():
    batch_clear()
    wls = _small_batch(n=12)
    eng = GpuEngine.instance()
    results, stats = eng.execute_batch([w.plan for w in wls], [w.inputs for w in wls],
                                       batch=BatchOptions(autotune=True))
    assert stats["block"] in (256, 512) and stats["tile_rows"] in (16384, 65536)
    for wl, r in zip(wls, results):
        _check_against_oracle(wl, r.columns)
