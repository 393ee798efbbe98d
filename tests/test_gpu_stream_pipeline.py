"""Stream pipeline (GpuStreamPipeline): batches of a projection chain with overlapped upload,
compute and download must give the same columns as the plain execution, bit-exact for integer work
(the reference pins a*2+b and a-b: cuda_engine/tests/test_gpu_stream_pipeline.cpp:201-290), in
submission order, with NULLs propagated."""
import numpy as np
import pytest

from vectisdb_b200 import GpuEngine, StreamPipeline, make_column, make_expr, make_projection, make_scan
from vectisdb_b200.engine import GpuValueType as T

pytestmark = pytest.mark.gpu


def _plan():
    scan = make_scan(["a", "b"])
    inner = make_projection([make_expr("((long long*)out)[idx] = ((const long long*)inputs[0])[row];", ["a"], T.INT64),
                             make_expr("((long long*)out)[idx] = ((const long long*)inputs[0])[row];", ["b"], T.INT64)],
                            scan)
    return make_projection([
        make_expr("((long long*)out)[idx] = ((const long long*)inputs[0])[row] * 2 + ((const long long*)inputs[1])[row];",
                  ["col0", "col1"], T.INT64),
        make_expr("((long long*)out)[idx] = ((const long long*)inputs[0])[row] - ((const long long*)inputs[1])[row];",
                  ["col0", "col1"], T.INT64)], inner)


def test_batches_match_plain_execution_in_order():
    rng = np.random.default_rng(1)
    plan = _plan()
    assert StreamPipeline.supports(plan)
    p = StreamPipeline(plan, ["a", "b"], [T.INT64, T.INT64], max_rows_per_batch=1 << 15, depth=3)
    assert p.output_types == [T.INT64, T.INT64]
    batches = []
    for i in range(12):
        n = (1 << 15) if i < 11 else 1234  # a short tail batch
        a = rng.integers(-(1 << 40), 1 << 40, n)
        b = rng.integers(-(1 << 40), 1 << 40, n)
        batches.append((a, b))
    got, pending = [], 0
    for a, b in batches:
        while not p.can_submit():
            got.append(p.take_blocking())
        p.submit([make_column("a", T.INT64, a), make_column("b", T.INT64, b)])
        a[:] = 0  # the caller's buffers are free once submit returns
        r = p.try_take()
        if r is not None:
            got.append(r)
        assert p.in_flight() <= 3
    while True:
        r = p.take_blocking()
        if r is None:
            break
        got.append(r)
    assert len(got) == len(batches)
    rng = np.random.default_rng(1)
    for (a_cleared, b), cols in zip(batches, got):
        n = len(b)
        a = rng.integers(-(1 << 40), 1 << 40, n)
        rng.integers(-(1 << 40), 1 << 40, n)
        assert np.array_equal(cols[0].data, a * 2 + b) and np.array_equal(cols[1].data, a - b)
        assert cols[0].name == "col0" and cols[1].name == "col1"
    p.close()


def test_nulls_propagate_and_unsupported_shapes_refused():
    plan = _plan()
    p = StreamPipeline(plan, ["a", "b"], [T.INT64, T.INT64], max_rows_per_batch=4096)
    a = np.arange(1000, dtype=np.int64)
    b = np.arange(1000, dtype=np.int64) * 3
    valid = np.ones(1000, bool)
    valid[::7] = False
    p.submit([make_column("a", T.INT64, a, validity=valid), make_column("b", T.INT64, b)])
    cols = p.take_blocking()
    assert np.array_equal(cols[0].validity, valid) and np.array_equal(cols[1].validity, valid)
    assert np.array_equal(cols[0].data[valid], (a * 2 + b)[valid])
    solo = GpuEngine.instance().execute_plan(plan, [make_column("a", T.INT64, a, validity=valid),
                                                    make_column("b", T.INT64, b)])
    assert np.array_equal(solo.columns[1].data[valid], cols[1].data[valid])
    with pytest.raises(Exception):
        p.submit([make_column("b", T.INT64, b), make_column("a", T.INT64, a)])  # names out of order
    p.close()
    from vectisdb_b200 import make_filter
    filt = make_filter([make_expr("((bool*)out)[idx] = ((const long long*)inputs[0])[row] > 0;", ["a"], T.BOOLEAN)],
                       make_scan(["a", "b"]))
    assert not StreamPipeline.supports(filt)
    with pytest.raises(Exception):
        StreamPipeline(filt, ["a", "b"], [T.INT64, T.INT64], 1024)


def test_running_sum_continues_across_batches():
    """RUNNING_SUM (the reference pipeline's window primitive, gpu_stream_pipeline.cu:133-166, 700-704):
    each value of a window column is that column's total over every row submitted so far, across batches
    of uneven sizes (one row, just below and above the 4096-row tile, several tiles). INT16 wraps in its
    width; the FLOAT64 inputs are multiples of 1/512 whose partial sums stay exact, so every column
    compares bit for bit. A batch with NULLs under a window column is refused and leaves the total as it
    was."""
    from vectisdb_b200.engine import GpuWindowPrimitive as W
    rng = np.random.default_rng(7)
    exprs = [make_expr("((long long*)out)[idx] = ((const long long*)inputs[0])[row];", ["a"], T.INT64),
             make_expr("((double*)out)[idx] = ((const double*)inputs[0])[row] * 2.0;", ["x"], T.FLOAT64),
             make_expr("((short*)out)[idx] = ((const short*)inputs[0])[row];", ["s"], T.INT16),
             make_expr("((long long*)out)[idx] = ((const long long*)inputs[0])[row];", ["a"], T.INT64)]
    for e in exprs[:3]:
        e.window_primitive = W.RUNNING_SUM
    plan = make_projection(exprs, make_scan(["a", "x", "s"]))
    assert StreamPipeline.supports(plan)
    p = StreamPipeline(plan, ["a", "x", "s"], [T.INT64, T.FLOAT64, T.INT16], max_rows_per_batch=20000, depth=3)
    sizes = [20000, 1, 4095, 4096, 4097, 12345, 1, 777]
    batches = [(rng.integers(-(1 << 40), 1 << 40, n), rng.integers(0, 1 << 20, n) / 1024.0,
                rng.integers(-32768, 32768, n).astype(np.int16)) for n in sizes]
    got = []
    for i, (a, x, s) in enumerate(batches):
        while not p.can_submit():
            got.append(p.take_blocking())
        if i == 5:  # a NULL under a window column: refused before it takes a stage
            with pytest.raises(Exception, match="RUNNING_SUM"):
                p.submit([make_column("a", T.INT64, a, np.arange(len(a)) != 3), make_column("x", T.FLOAT64, x),
                          make_column("s", T.INT16, s)])
        p.submit([make_column("a", T.INT64, a), make_column("x", T.FLOAT64, x), make_column("s", T.INT16, s)])
    while True:
        r = p.take_blocking()
        if r is None:
            break
        got.append(r)
    assert len(got) == len(batches)
    a_all = np.concatenate([b[0] for b in batches])
    x_all = np.concatenate([b[1] for b in batches])
    s_all = np.concatenate([b[2] for b in batches])
    want = [np.cumsum(a_all), np.cumsum(x_all * 2.0), np.cumsum(s_all.astype(np.int64)).astype(np.int16), a_all]
    at = 0
    for (a, _, _), cols in zip(batches, got):
        n = len(a)
        for c, w in zip(cols, want):
            assert c.data.dtype == w.dtype and np.array_equal(c.data, w[at:at + n]), (c.name, at, n)
        at += n
