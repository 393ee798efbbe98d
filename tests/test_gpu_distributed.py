"""sharded_group_by over the engine itself (one gloo rank): the plan rewritten for sharding (AVG as SUM
plus COUNT(*)), run by the engine, merged and finished on the host, must equal the engine's own run of
the original plan -- keys, counts, MIN/MAX and 128-bit sums bit for bit, AVG over DOUBLE within 1e-12
relative (the engine's FP64 sums are order-dependent). C0's 1024 keys take the dense merge; C1's two
keys (about 24 packed bits) take the hash repartition, merged in numpy or re-aggregated by the engine
(its GROUP BY over the exchanged partial columns)."""
import datetime
import socket

import numpy as np
import pytest

from vectisdb_b200 import GpuEngine
from vectisdb_b200 import workloads as W
from vectisdb_b200.engine import GpuAggregateKind as A, GpuValueType as T, HUGEINT_DTYPE

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def one_rank():
    import torch.distributed as dist
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    yield
    dist.destroy_process_group()


def _compare(plan, inputs, column_types, reaggregate=None):
    from vectisdb_b200.distributed import sharded_group_by
    eng = GpuEngine.instance()
    direct = eng.execute_plan(plan, inputs)
    assert direct.success, direct.error_message
    nk = len(plan.group_keys)
    keys = [c.data for c in direct.columns[:nk]]
    order = np.lexsort(tuple(reversed(keys)))  # first key first, as sharded_group_by returns them

    def run_local(p):
        r = eng.execute_plan(p, inputs)
        assert r.success, r.error_message
        return r.columns

    got = sharded_group_by(plan, run_local, column_types, reaggregate=reaggregate)
    assert [n for n, _ in got] == list(plan.group_keys) + [f"agg_{i}" for i in range(len(plan.aggregates))]
    for (name, g), c in zip(got, direct.columns):
        want = c.data[order]
        assert g.dtype == want.dtype and len(g) == len(want), name
        i = list(plan.group_keys).index(name) if name in plan.group_keys else None
        agg = None if i is not None else plan.aggregates[int(name[4:])]
        if agg is not None and agg.kind in (A.AVG, A.SUM) and agg.output_type == T.FLOAT64:
            assert np.all(np.abs(g - want) <= 1e-12 * np.abs(want)), name
        elif g.dtype == HUGEINT_DTYPE:
            assert np.array_equal(g["lower"], want["lower"]) and np.array_equal(g["upper"], want["upper"]), name
        else:
            assert np.array_equal(g, want), name
    return len(keys[0])


def test_dense_keys_through_the_engine(one_rank):
    wl = W.c0(n=1 << 18)
    assert _compare(wl.plan, wl.inputs, {}) == 1024


def test_high_cardinality_keys_and_avg_through_the_engine(one_rank):
    wl = W.c1(n=1 << 18)
    groups = _compare(wl.plan, wl.inputs, {"v": T.FLOAT64})
    assert groups > (1 << 14)


def test_high_cardinality_merge_re_aggregated_by_the_engine(one_rank):
    """The repartitioned partial groups merged by the engine's own GROUP BY (128-bit sums as exact
    32-bit chunk sums, counts as 128-bit sums, float MIN/MAX as order-preserving integers)."""
    wl = W.c1(n=1 << 18)
    eng = GpuEngine.instance()
    calls = []

    def reaggregate(p, cols):
        calls.append(len(cols))
        r = eng.execute_plan(p, cols)
        assert r.success, r.error_message
        return r.columns

    groups = _compare(wl.plan, wl.inputs, {"v": T.FLOAT64}, reaggregate)
    assert groups > (1 << 14) and len(calls) == 1
