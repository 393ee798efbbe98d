"""Result handoff in DuckDB's STANDARD_VECTOR_SIZE chunks through vgpu_result_column_range (the
reference's PhysicalGpuExecute::GetData emission, extension/src/physical_gpu_execute.cpp:506-517): the
chunks are views into the result (no copy) that concatenate to the whole result -- NULL bits included,
as DuckDB's 64-bit validity words -- and HUGEINT sums arrive in hugeint_t layout; slicing a column with
validity off a 64-row boundary is refused."""
import numpy as np
import pytest

from vectisdb_b200 import GpuEngine, make_aggregate, make_column, make_expr, make_filter, make_group_by, make_scan
from vectisdb_b200.engine import GpuAggregateKind as A, GpuValueType as T, hugeint_to_int

pytestmark = pytest.mark.gpu


def test_filtered_rows_with_nulls_in_2048_row_chunks():
    rng = np.random.default_rng(44)
    n = 20_000
    k = rng.integers(0, 100, n).astype(np.int32)
    lv = rng.integers(-10**12, 10**12, n).astype(np.int64)
    valid = rng.random(n) > 0.1
    plan = make_filter([make_expr("((bool*)out)[idx] = (((const int*)inputs[0])[row] % 3) != 0;", ["k"], T.BOOLEAN)],
                       make_scan(["k", "lv"]))
    inputs = [make_column("k", T.INT32, k), make_column("lv", T.INT64, lv, valid)]
    eng = GpuEngine.instance()
    whole = eng.execute_plan(plan, inputs)
    assert whole.success, whole.error_message
    rows = len(whole.columns[0].data)
    chunks = list(eng.execute_plan_chunks(plan, inputs))
    assert len(chunks) == (rows + 2047) // 2048 and all(len(c[0][0]) == 2048 for c in chunks[:-1])
    assert np.array_equal(np.concatenate([c[0][0] for c in chunks]), whole.columns[0].data)
    got = np.concatenate([c[1][0] for c in chunks])
    bits = np.concatenate([np.unpackbits(c[1][1].view(np.uint8), bitorder="little")[: len(c[1][0])] for c in chunks])
    want = np.asarray(whole.columns[1].validity, np.uint8)  # per-row validity of the host result
    assert np.array_equal(bits, want) and not bits.all()
    keep = bits.astype(bool)
    assert np.array_equal(got[keep], whole.columns[1].data[keep])
    assert all(c[0][1] is None for c in chunks)  # k has no NULLs: no validity words
    with pytest.raises(ValueError):
        next(eng.execute_plan_chunks(plan, inputs, chunk_rows=1000))


def test_hugeint_sums_in_chunks():
    rng = np.random.default_rng(45)
    n = 50_000
    g = rng.integers(0, 5000, n).astype(np.int32)
    x = rng.integers((1 << 62) - 100, 1 << 62, n).astype(np.int64)
    plan = make_group_by(["g"], [make_aggregate(A.SUM, "x", T.HUGEINT)], make_scan(["g", "x"]))
    inputs = [make_column("g", T.INT32, g), make_column("x", T.INT64, x)]
    chunks = list(GpuEngine.instance().execute_plan_chunks(plan, inputs))
    keys = np.concatenate([c[0][0] for c in chunks])
    sums = hugeint_to_int(np.concatenate([c[1][0] for c in chunks]))
    assert len(keys) == len(np.unique(g))
    for key, s in zip(keys.tolist()[:200], sums[:200]):
        assert s == int(x[g == key].astype(object).sum())
