"""Serving: requests admitted against a device-memory budget run concurrently (and same-template
group-bys in one batched launch); each result must be the one the request gives alone (integer and
COUNT/MIN/MAX bit-exact, FP64 within 1e-12 relative)."""
import numpy as np
import pytest

from vectisdb_b200 import GpuEngine, Server
from vectisdb_b200 import workloads as W

pytestmark = pytest.mark.gpu

REL = 1e-12


def _rows(cols, nkeys):
    keys = [np.asarray(c.data) for c in cols[:nkeys]]
    order = np.lexsort(tuple(reversed(keys))) if keys else np.arange(cols[0].row_count)
    return [np.asarray(c.data)[order] for c in cols]


def _same(a, b, nkeys):
    assert len(a.columns) == len(b.columns)
    ra, rb = _rows(a.columns, nkeys), _rows(b.columns, nkeys)
    for x, y in zip(ra, rb):
        assert len(x) == len(y)
        if x.dtype.kind == "f":
            assert np.all(np.abs(x - y) <= REL * np.maximum(np.abs(y), 1e-300))
        else:
            assert np.array_equal(x, y)


def _mix(seed=11):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(24):
        kind = rng.choice(["c0", "c0", "c1", "c2"])
        n = int(2 ** rng.uniform(12, 17))
        if kind == "c0":
            wl = W.c0(n=n, seed=1000 + i, k_card=int(rng.integers(16, 2048)), v_lt=float(rng.uniform(0.2, 0.8)),
                      w_mod=int(rng.integers(2, 13)))
            reqs.append((wl, 1))
        elif kind == "c1":
            reqs.append((W.c1(n=n, seed=2000 + i), 2))
        else:
            reqs.append((W.c2(probe_n=n, build_n=1 << 12, miss_lo=1 << 12, miss_span=1 << 12, seed=3000 + i), 1))
    return reqs


@pytest.mark.parametrize("slots,batch_max", [(4, 64), (1, 1)])
def test_each_result_same_alone_and_in_the_mix(slots, batch_max):
    eng = GpuEngine.instance()
    reqs = _mix()
    alone = [eng.execute_plan(wl.plan, wl.inputs) for wl, _ in reqs]
    srv = Server(slots=slots, batch_max=batch_max)
    ids = [srv.submit(wl.plan, wl.inputs) for wl, _ in reqs]
    for rid, (wl, nkeys), solo in zip(ids, reqs, alone):
        res, info = srv.wait(rid)
        assert info["status"] == 0, info["error"]
        _same(res, solo, nkeys)
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    if slots > 1:
        assert st["batches"] >= 1 and st["batched_requests"] >= 2  # C0 requests of one template batched
    else:
        assert st["peak_in_flight"] == 1 and st["batches"] == 0
    srv.close()


def test_admission_respects_the_memory_budget_and_rejects_oversized():
    eng = GpuEngine.instance()
    reqs = [(W.c1(n=1 << 16, seed=50 + i), 2) for i in range(8)]
    srv = Server(slots=4, batch_max=1)
    # learn one request's estimate, then size the budget for about two at a time
    rid = srv.submit(reqs[0][0].plan, reqs[0][0].inputs)
    _, info = srv.wait(rid)
    est = info["estimated_bytes"]
    srv.close()
    srv = Server(slots=4, batch_max=1, memory_budget_bytes=int(2.5 * est))
    ids = [srv.submit(wl.plan, wl.inputs) for wl, _ in reqs]
    big = W.c1(n=1 << 20, seed=99)
    big_id = srv.submit(big.plan, big.inputs)
    for rid, (wl, nkeys) in zip(ids, reqs):
        res, info = srv.wait(rid)
        assert info["status"] == 0, info["error"]
        _same(res, eng.execute_plan(wl.plan, wl.inputs), nkeys)
    res, info = srv.wait(big_id)
    assert res is None and info["status"] != 0 and "admission budget" in info["error"]
    st = srv.stats()
    assert st["peak_reserved_bytes"] <= st["budget_bytes"] and st["peak_in_flight"] <= 2
    assert st["rejected"] == 1
    srv.close()
