"""The C-ABI library loads without a GPU and exports every function include/vgpu.h declares."""
import ctypes as C

import numpy as np

from vectisdb_b200 import abi
from vectisdb_b200.engine import sha256_hex


def test_library_exports_every_declared_symbol():
    lib = abi.lib()
    declared = abi.declared_functions()
    assert len(declared) >= 30
    missing = [name for name in declared if not hasattr(lib, name)]
    assert not missing, missing
    bound = {name for name, _, _ in abi.SIGNATURES}
    assert set(declared) == bound, set(declared) ^ bound


def test_abi_version_and_status_strings():
    lib = abi.lib()
    assert lib.vgpu_abi_version() == abi.ABI_VERSION
    assert lib.vgpu_status_string(abi.ERR_UNSUPPORTED) == b"UNSUPPORTED"


def test_sha256_known_vectors():
    # KernelCache::HashSource known answers (cuda_engine/tests/test_kernel_cache.cpp:68-75)
    assert sha256_hex(b"") == "e3b0c44298fc1c149afbf4c8996fb92427ae41e4649b934ca495991b7852b855"
    assert sha256_hex(b"abc") == "ba7816bf8f01cfea414140de5dae2223b00361a396177a9cb410ff61f20015ad"
    assert len(sha256_hex(b"x")) == 64
    assert sha256_hex(b"out[idx] = a + b;") != sha256_hex(b"out[idx] = a - b;")
    long = bytes(range(256)) * 17
    import hashlib
    assert sha256_hex(long) == hashlib.sha256(long).hexdigest()


def test_malformed_plans_fail_cleanly_without_a_device():
    lib = abi.lib()
    res = C.c_void_p()
    # empty plan
    plan = abi.vgpu_plan()
    assert lib.vgpu_execute_plan(C.byref(plan), None, 0, None, C.byref(res)) == abi.ERR_INVALID_ARGUMENT
    assert b"empty plan" in lib.vgpu_last_error()
    # child index out of range
    nodes = (abi.vgpu_plan_node * 1)()
    kids = (C.c_uint32 * 1)(5)
    nodes[0].op = 1
    nodes[0].n_children = 1
    nodes[0].children = C.cast(kids, C.POINTER(C.c_uint32))
    plan = abi.vgpu_plan(C.cast(nodes, C.POINTER(abi.vgpu_plan_node)), 1, 0)
    assert lib.vgpu_execute_plan(C.byref(plan), None, 0, None, C.byref(res)) == abi.ERR_INVALID_ARGUMENT
    # a cycle
    kids[0] = 0
    assert lib.vgpu_execute_plan(C.byref(plan), None, 0, None, C.byref(res)) == abi.ERR_INVALID_ARGUMENT
    assert b"cycle" in lib.vgpu_last_error()
    # unknown op
    nodes[0].op = 99
    nodes[0].n_children = 0
    assert lib.vgpu_execute_plan(C.byref(plan), None, 0, None, C.byref(res)) == abi.ERR_INVALID_ARGUMENT
    assert not res.value


def test_row_independence_and_working_set():
    from vectisdb_b200 import workloads as W
    from vectisdb_b200.engine import estimate_working_set, is_row_independent, make_expr, make_projection, make_scan
    from vectisdb_b200.engine import GpuValueType as T
    assert not is_row_independent(W.c0_plan())
    p = make_projection([make_expr("((int*)out)[idx] = ((const int*)inputs[0])[row];", ["k"], T.INT32)],
                        make_scan(["k"]))
    assert is_row_independent(p)
    plan = W.c1_plan(0)
    plan.children[0].children[0].estimated_rows = 1 << 27
    plan.children[0].children[0].estimated_row_width_bytes = 32
    ws = estimate_working_set(plan)
    assert ws.total_bytes >= (1 << 27) * 32
    assert ws.largest_operator in (b"GROUP_BY_AGGREGATE", b"SCAN")


def test_working_set_formulas():
    """The working-set estimate (csrc/cost_model.cpp), pinned on hand-computed plans. It charges what the
    executor allocates: host scans are copied (rows x width); a FILTER/PROJECTION chain, and a join or
    cross product under one, is one fused pipeline that allocates only where its rows are materialized
    (the root, a join's build side); a GROUP BY whose state fits the one-pass strategy allocates per group,
    otherwise one 32-byte-aligned record per input row plus outputs per group, partition offsets and
    split-partition tables; a fused join its build-side table, a materializing join its key, search and
    index buffers and outputs; a root cross product every pair. Sizes saturate instead of wrapping."""
    from vectisdb_b200.engine import (GpuAggregateKind as A, GpuValueType as T, estimate_working_set, make_aggregate,
                                      make_cross_product, make_expr, make_filter, make_group_by, make_join,
                                      make_projection, make_scan)
    scan = make_scan(["k", "v", "w"])
    scan.estimated_rows, scan.estimated_row_width_bytes = 1000, 20
    filt = make_filter([make_expr("out[idx] = 1;", ["v"], T.BOOLEAN)], scan)
    gb = make_group_by(["k"], [make_aggregate(A.SUM, "v", T.FLOAT64), make_aggregate(A.COUNT_STAR, "", T.INT64)], filt)
    ws = estimate_working_set(gb)
    scan_b = 1000 * 20
    gb_b = 1000 * (2 * 8 + (8 + 8 + 8)) + 64  # one pass: state words (COUNT, SUM) + key/SUM/COUNT outputs
    assert ws.total_bytes == scan_b + gb_b  # the filter streams into the group-by: nothing of its own
    assert ws.largest_bytes == gb_b and ws.largest_operator == b"GROUP_BY_AGGREGATE" and not ws.chunk_capped

    many = make_scan(["a", "b", "amt", "v", "ts"])
    many.estimated_rows, many.estimated_row_width_bytes = 1 << 20, 32
    hc = make_group_by(["a", "b"], [make_aggregate(A.SUM, "amt", T.HUGEINT), make_aggregate(A.AVG, "v", T.FLOAT64),
                                    make_aggregate(A.COUNT_STAR, "", T.INT64), make_aggregate(A.MAX, "ts", T.INT64)],
                       many)
    hc.estimated_rows = 300_000  # groups
    ws = estimate_working_set(hc)
    fields = 1 + 2 + 1 + 1  # COUNT, 128-bit SUM, FP64 sum of AVG, MAX
    hc_b = ((1 << 20) * 32 + 300_000 * (16 + 16 + 8 + 8 + 8) + min(16384 * 2048 * 4 // 8, (1 << 20) * 8)
            + fields * 8 * 4096 * min(4 * 148, (1 << 20) // 16384 + 1))
    assert ws.total_bytes == (1 << 20) * 32 + hc_b

    big = make_scan(["k"])
    big.estimated_rows, big.estimated_row_width_bytes = 1_000_000, 4
    proj = make_projection([make_expr("((int*)out)[idx] = ((const int*)inputs[0])[row];", ["k"], T.INT32)], big)
    ws = estimate_working_set(proj, max_chunk_rows=1000)  # row-independent: charged one chunk at a time
    assert ws.chunk_capped and ws.total_bytes == 1000 * 4 + (1000 * 4 + 1000 // 256 + 64)

    left, right = make_scan(["a", "x"]), make_scan(["b", "g"])
    left.estimated_rows, left.estimated_row_width_bytes = 100, 16
    right.estimated_rows, right.estimated_row_width_bytes = 50, 12
    join = make_join("a", "b", ["a", "x", "g"], left, right)
    ws = estimate_working_set(join)  # at the root: materializing
    join_b = 100 * 24 + 50 * 24 + 100 * (3 * 8 + 8)
    assert ws.total_bytes == 1600 + 600 + join_b and ws.largest_operator == b"HASH_JOIN"
    fused = make_group_by(["g"], [make_aggregate(A.SUM, "x", T.FLOAT64)], make_join("a", "b", ["g", "x"], left, right))
    ws = estimate_working_set(fused)  # under a group-by: the join is the pipeline's source
    assert ws.total_bytes == 1600 + 600 + 50 * 32 + (100 * (2 * 8 + 16) + 64)

    l2, r2 = make_scan(["a"]), make_scan(["b"])
    l2.estimated_rows, l2.estimated_row_width_bytes = 10, 4
    r2.estimated_rows, r2.estimated_row_width_bytes = 20, 4
    ws = estimate_working_set(make_cross_product(["a", "b"], l2, r2))
    assert ws.total_bytes == 40 + 80 + 200 * 16 and ws.largest_operator == b"CROSS_PRODUCT"
    pred = make_filter([make_expr("out[idx] = 1;", ["a", "b"], T.BOOLEAN)], make_cross_product(["a", "b"], l2, r2))
    pred.estimated_rows = 15
    ws = estimate_working_set(pred)  # the pairs stay virtual; the filter materializes what passes
    assert ws.total_bytes == 40 + 80 + 15 * 16 + 15 // 256 + 64 and ws.largest_operator == b"FILTER"

    huge = make_scan(["k"])
    huge.estimated_rows, huge.estimated_row_width_bytes = 1 << 62, 8
    ws = estimate_working_set(make_filter([make_expr("out[idx] = 1;", ["k"], T.BOOLEAN)], huge))
    assert ws.total_bytes == (1 << 64) - 1


def test_working_set_for_inputs_skips_borrowed_scans():
    """With the execution's actual inputs, a scan over device-memory columns is borrowed (no charge),
    host columns are copied (rows x width from the inputs, not from the plan's estimates)."""
    import numpy as np
    from vectisdb_b200.engine import (GpuColumn, GpuValueType as T, estimate_working_set_for, make_column, make_expr,
                                      make_projection, make_scan)
    proj = make_projection([make_expr("((double*)out)[idx] = ((const double*)inputs[0])[row] * 2.0;", ["v"],
                                      T.FLOAT64)], make_scan(["v"]))
    host = make_column("v", T.FLOAT64, np.zeros(5000))
    ws = estimate_working_set_for(proj, [host])
    assert ws.total_bytes == 5000 * 8 + (5000 * 8 + 5000 // 256 + 64)
    dev = GpuColumn("v", T.FLOAT64, None, None, 5000, 0x1000)  # a device pointer is only described, never read
    ws = estimate_working_set_for(proj, [dev])
    assert ws.total_bytes == 5000 * 8 + 5000 // 256 + 64


def test_row_independence_by_operator():
    """Scans, projections and filters are row-wise (a chunk can run alone); a group-by, join or cross
    product anywhere below the root makes the plan need its input whole (cost model IsRowIndependent)."""
    from vectisdb_b200.engine import (GpuAggregateKind as A, GpuValueType as T, is_row_independent, make_aggregate,
                                      make_cross_product, make_expr, make_filter, make_group_by, make_join,
                                      make_projection, make_scan)
    e = make_expr("out[idx] = 1;", ["a"], T.BOOLEAN)
    assert is_row_independent(make_scan(["a"]))
    assert is_row_independent(make_filter([e], make_projection([e], make_filter([e], make_scan(["a"])))))
    gb = make_group_by(["a"], [make_aggregate(A.COUNT_STAR, "", T.INT64)], make_scan(["a"]))
    assert not is_row_independent(gb)
    assert not is_row_independent(make_filter([e], gb))
    assert not is_row_independent(make_projection([e], make_join("a", "b", ["a"], make_scan(["a"]), make_scan(["b"]))))
    assert not is_row_independent(make_cross_product(["a", "b"], make_scan(["a"]), make_scan(["b"])))


def test_plan_shape_columns_size_and_execution_mode():
    """The routing helpers the extension's table checker calls, pinned on hand-computed plans: a
    FILTER's price runs over the rows entering it, other nodes' over their own rows; nothing priced is
    INCONCLUSIVE; below 3 ops per scanned row INSUFFICIENT, from 10 SUFFICIENT; a plan that scans nothing
    keeps its numerators; a SCAN of width 0 counts 8 bytes per row; the uncached mode starts strictly
    above budget x threshold."""
    from vectisdb_b200.engine import (GpuAggregateKind as A, GpuExecutionMode as M, GpuValueType as T,
                                      GpuWorkDensity as D, analyze_plan_shape, determine_execution_mode,
                                      estimate_columns_size, make_aggregate, make_cross_product, make_expr,
                                      make_filter, make_group_by, make_join, make_projection, make_scan,
                                      serialize_plan_memo)

    def chain(filter_prices, projection_price):
        scan = make_scan(["a", "b"])
        scan.estimated_rows, scan.estimated_row_width_bytes = 1000, 16
        filt = make_filter([make_expr("out[idx] = 1;", ["a"], T.BOOLEAN, p) for p in filter_prices], scan)
        filt.estimated_rows = 300
        proj = make_projection([make_expr("out[idx] = 1;", ["a"], T.FLOAT64, projection_price)], filt)
        proj.estimated_rows = 300
        return proj

    s = analyze_plan_shape(chain([2.0, 3.0], 4.0))
    assert (s.scanned_rows, s.scanned_bytes, s.max_rows) == (1000, 16000, 1000)
    assert s.total_ops == 5 * 1000 + 4 * 300 and s.ops_per_scanned_row == 6.2
    assert s.ops_per_scanned_byte == 6200 / 16000 and s.amplification == 1.0 and s.density == D.INCONCLUSIVE
    assert analyze_plan_shape(chain([2.0, 3.0], 40.0)).density == D.SUFFICIENT  # 17 ops per row
    assert analyze_plan_shape(chain([2.0, 3.0], 50.0 / 3.0)).density == D.SUFFICIENT  # exactly 10
    s = analyze_plan_shape(chain([1.0], 0.0))
    assert s.ops_per_scanned_row == 1.0 and s.density == D.INSUFFICIENT

    left, right = make_scan(["a"]), make_scan(["b"])
    left.estimated_rows, right.estimated_rows = 100, 90
    cross = make_cross_product(["a", "b"], left, right)
    cross.estimated_rows = 9000
    gb = make_group_by(["a"], [make_aggregate(A.COUNT_STAR, "", T.INT64)], cross)
    gb.estimated_rows = 5
    s = analyze_plan_shape(gb)  # unpriced: unmeasured, not cheap
    assert s.total_ops == 0 and s.density == D.INCONCLUSIVE
    assert s.scanned_bytes == 190 * 8 and s.amplification == 9000 / 190
    assert estimate_columns_size(gb) == 1520

    empty = make_scan(["a"])
    proj = make_projection([make_expr("out[idx] = 1;", ["a"], T.FLOAT64, 2.0)], empty)
    proj.estimated_rows = 10
    s = analyze_plan_shape(proj)
    assert s.scanned_rows == 0 and s.total_ops == 20 and s.ops_per_scanned_row == 20
    assert s.ops_per_scanned_byte == 20 and s.amplification == 10 and s.density == D.SUFFICIENT

    l2, r2 = make_scan(["a", "x"]), make_scan(["b"])
    l2.estimated_rows, l2.estimated_row_width_bytes, r2.estimated_rows = 100, 16, 50
    join = make_join("a", "b", ["a", "x"], l2, r2)
    assert estimate_columns_size(join) == 100 * 16 + 50 * 8
    assert determine_execution_mode(join, 0) == M.PIPELINE_STREAM_CACHED  # no budget: never uncached
    assert determine_execution_mode(join, 2000) == M.PIPELINE_STREAM_UNCACHED  # 2000 > 1500
    assert determine_execution_mode(join, 4000) == M.PIPELINE_STREAM_CACHED  # 2000 <= 3000
    assert determine_execution_mode(join, 2000, 1.0) == M.PIPELINE_STREAM_CACHED  # strictly above

    plan = chain([2.0], 4.0)  # the serialized-plan memo notices a changed price
    first, _ = serialize_plan_memo(plan)
    plan.expressions[0].estimated_ops_per_row = 5.0
    again, _ = serialize_plan_memo(plan)
    assert again is not first and again.nodes[again.root].expressions[0].estimated_ops_per_row == 5.0


def test_running_sum_window_expressions_reach_only_the_stream_pipeline():
    """A RUNNING_SUM window expression (GpuExpr::window_primitive) crosses the boundary intact. The
    stream pipeline takes it on top-level numeric outputs only; plain execution refuses it with
    VGPU_ERR_UNSUPPORTED before any device work, instead of returning a plain projection's values. An
    out-of-range primitive is a malformed plan. Routing helpers still read the plan."""
    from vectisdb_b200.engine import (GpuValueType as T, GpuWindowPrimitive as W, StreamPipeline, _Keep,
                                      estimate_columns_size, make_expr, make_projection, make_scan, serialize_plan)
    lib = abi.lib()
    e = make_expr("((double*)out)[idx] = ((const double*)inputs[0])[row];", ["x"], T.FLOAT64)
    e.window_primitive = W.RUNNING_SUM
    plan = make_projection([e], make_scan(["x"]))
    keep = _Keep()
    plan_c = serialize_plan(plan, keep)
    assert plan_c.nodes[plan_c.root].expressions[0].window_primitive == 1
    res = C.c_void_p()
    assert lib.vgpu_execute_plan(C.byref(plan_c), None, 0, None, C.byref(res)) == abi.ERR_UNSUPPORTED
    assert b"RUNNING_SUM" in lib.vgpu_last_error() and not res.value
    assert StreamPipeline.supports(plan)  # top level, DOUBLE
    above = make_projection([make_expr("((double*)out)[idx] = ((const double*)inputs[0])[row];", ["col0"], T.FLOAT64)],
                            plan)
    assert not StreamPipeline.supports(above)  # a running total below the top level
    b = make_expr("((bool*)out)[idx] = ((const double*)inputs[0])[row] > 0;", ["x"], T.BOOLEAN)
    b.window_primitive = W.RUNNING_SUM
    assert not StreamPipeline.supports(make_projection([b], make_scan(["x"])))  # not a numeric output
    plan.children[0].estimated_rows = 10
    assert estimate_columns_size(plan) == 80
    plan_c = serialize_plan(plan, keep)
    plan_c.nodes[plan_c.root].expressions[0].window_primitive = 7
    assert lib.vgpu_execute_plan(C.byref(plan_c), None, 0, None, C.byref(res)) == abi.ERR_INVALID_ARGUMENT
    assert b"window primitive" in lib.vgpu_last_error()


def test_aggregate_descriptors_cross_the_boundary_and_are_checked():
    """GpuPlanNode::aggregate_exprs: none, or one descriptor per aggregate (the reference's group-by
    refuses any other count); the descriptors are carried, never executed."""
    from vectisdb_b200.engine import (GpuAggregateKind as A, GpuValueType as T, _Keep, estimate_working_set,
                                      make_aggregate, make_group_by, make_scan, serialize_plan)
    lib = abi.lib()
    gb = make_group_by(["k"], [make_aggregate(A.COUNT_STAR, "", T.INT64), make_aggregate(A.SUM, "v", T.FLOAT64)],
                       make_scan(["k", "v"]))
    estimate_working_set(gb)  # no descriptors: fine
    gb.aggregate_exprs = ["count_star()", "sum(v)"]
    keep = _Keep()
    plan_c = serialize_plan(gb, keep)
    node = plan_c.nodes[plan_c.root]
    assert node.n_aggregate_exprs == 2 and node.aggregate_exprs[1] == b"sum(v)"
    estimate_working_set(gb)  # one per aggregate: fine
    gb.aggregate_exprs = ["count_star()"]
    res = C.c_void_p()
    assert lib.vgpu_execute_plan(C.byref(serialize_plan(gb, keep)), None, 0, None, C.byref(res)) == abi.ERR_INVALID_ARGUMENT
    assert b"disagree in length" in lib.vgpu_last_error()
