"""Host ingest: the conversion of DuckDB-shaped vectors (vgpu_convert_vector, no device needed) follows
the reference's vector_converter (extension/src/vector_converter.cpp:87-273) -- flat, dictionary
(selection vector) and constant vectors, validity by physical index, an optional row selection on
top, a bitmap only when a NULL is met; and (on the GPU) chunks appended to an ingest handle land in the
column cache exactly, NULLs included, across batch boundaries, as a table queries then read."""
import numpy as np
import pytest

from vectisdb_b200 import abi
from vectisdb_b200.engine import GpuValueType as T
from vectisdb_b200.ingest import Vector, convert_vector, validity_words


def _bits(bitmap, n):
    return np.unpackbits(bitmap, bitorder="little")[:n].astype(bool)


def test_flat_vector_without_nulls_has_no_bitmap():
    x = np.arange(100, dtype=np.int64) * 3
    out, bm = convert_vector(Vector(x), T.INT64, 100)
    assert np.array_equal(out, x) and bm is None


def test_dictionary_vector_reads_through_its_selection():
    dict_values = np.array([1.5, -2.0, 7.25], dtype=np.float64)
    sel = np.array([2, 0, 0, 1, 2, 1], dtype=np.uint32)
    out, bm = convert_vector(Vector(dict_values, sel=sel), T.FLOAT64, 6)
    assert np.array_equal(out, dict_values[sel]) and bm is None


def test_constant_vector_repeats_its_value_for_every_row():
    out, bm = convert_vector(Vector(np.array([42], np.int32), constant=True), T.INT32, 2048)
    assert np.array_equal(out, np.full(2048, 42, np.int32)) and bm is None
    out, bm = convert_vector(Vector(np.array([42], np.int32), constant=True, validity=validity_words([False])),
                             T.INT32, 5)
    assert bm is not None and not _bits(bm, 5).any()  # a NULL constant: every row NULL


def test_validity_is_by_physical_index_and_row_selection_applies_first():
    phys = np.arange(10, dtype=np.int16)
    valid = np.ones(10, bool)
    valid[[3, 7]] = False
    sel = np.array([9, 7, 3, 3, 0, 1], np.uint32)          # logical -> physical
    row_sel = np.array([0, 1, 2, 5], np.uint32)             # rows of the chunk kept
    out, bm = convert_vector(Vector(phys, sel=sel, validity=validity_words(valid)), T.INT16, 4, row_sel)
    assert np.array_equal(out, phys[sel[row_sel]])
    assert np.array_equal(_bits(bm, 4), valid[sel[row_sel]])


def test_unsupported_types_are_refused():
    with pytest.raises(abi.VgpuError) as e:
        convert_vector(Vector(np.zeros(4, np.int32)), T.DICTIONARY_STRING, 4)
    assert e.value.status == abi.ERR_UNSUPPORTED


@pytest.mark.gpu
def test_chunks_land_in_the_column_cache_across_batches():
    from vectisdb_b200 import ColumnCache, ExecuteOptions, GpuEngine, GpuTableRef, make_aggregate, make_group_by, make_scan
    from vectisdb_b200.engine import GpuAggregateKind as A
    from vectisdb_b200.ingest import TableIngest
    rng = np.random.default_rng(4)
    n_chunks, chunk = 37, 2048
    k = rng.integers(0, 100, n_chunks * chunk).astype(np.int32)
    v = rng.random(n_chunks * chunk)
    w = rng.integers(-10**9, 10**9, n_chunks * chunk).astype(np.int64)
    w_valid = rng.random(n_chunks * chunk) > 0.05
    t = GpuTableRef("memory", "main", "ingested")
    kept = np.zeros(0, np.int64)
    try:
        with TableIngest(t, [("k", T.INT32), ("v", T.FLOAT64), ("w", T.INT64)], batch_rows=10_000) as ing:
            for c in range(n_chunks):
                lo = c * chunk
                sel = None
                rows = np.arange(lo, lo + chunk)
                if c % 5 == 3:  # a filtered chunk: the scan's row selection
                    sel = np.flatnonzero(rng.random(chunk) > 0.4).astype(np.uint32)
                    rows = lo + sel
                if c % 7 == 2:  # a dictionary-encoded k vector
                    dvals = np.unique(k[lo:lo + chunk])
                    kv = Vector(dvals, sel=np.searchsorted(dvals, k[lo:lo + chunk]).astype(np.uint32))
                else:
                    kv = Vector(k[lo:lo + chunk])
                ing.append([kv, Vector(v[lo:lo + chunk]), Vector(w[lo:lo + chunk], validity=validity_words(w_valid[lo:lo + chunk]))],
                           len(rows) if sel is not None else chunk, sel)
                kept = np.concatenate([kept, rows])
        r = GpuEngine.instance().execute_plan(make_scan(["k", "v", "w"], t), [], ExecuteOptions(serve_whole_scan_from_cache=True))
        assert r.success, r.error_message
        gk, gv, gw = r.columns
        assert np.array_equal(gk.data, k[kept]) and np.array_equal(gv.data, v[kept])
        valid = w_valid[kept]
        assert np.array_equal(np.asarray(gw.validity, bool), valid)  # per-row validity of the host result
        assert np.array_equal(gw.data[valid], w[kept][valid])
        plan = make_group_by(["k"], [make_aggregate(A.COUNT_STAR, "", T.INT64)], make_scan(["k"], t))
        r = GpuEngine.instance().execute_plan(plan, [], ExecuteOptions(serve_whole_scan_from_cache=True))
        assert r.success, r.error_message
        got = dict(zip(r.columns[0].data.tolist(), r.columns[1].data.tolist()))
        want = dict(zip(*np.unique(k[kept], return_counts=True)))
        assert got == {int(a): int(b) for a, b in want.items()}
    finally:
        ColumnCache.invalidate_table(t)
