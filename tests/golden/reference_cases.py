"""The known-answer cases of the reference engine's test suite, re-expressed over this engine's API.

Each case rebuilds the plan and the deterministic inputs of one test in
cuda_engine/tests/test_gpu_executor.cpp (cited per case) and states the reference test's own
expectation: the rows it checks (computed by the same CPU loops the test uses), the comparison it
makes (positional order, group set, or row multiset) and, for refusals, the substring it requires in
the error message. make_golden.py evaluates `expected()` once and writes reference_cases.json; the
tests compare both the oracle and the GPU engine against that file.
"""
from __future__ import annotations

from collections import defaultdict

import numpy as np

from vectisdb_b200.engine import (GpuAggregateKind as A, GpuValueType as T, make_aggregate, make_column,
                                  make_cross_product, make_expr, make_filter, make_group_by, make_join,
                                  make_projection, make_scan)

CASES = {}


def case(line):
    def deco(fn):
        CASES[fn.__name__] = (line, fn)
        return fn
    return deco


def expr(body, inputs, t):
    return make_expr(body, inputs, t)


def rows_of(*cols):
    return [list(r) for r in zip(*cols)]


def ok(rows, compare, keys=0, float_tol=0.0, null_values_checked=False):
    """rows: expected output rows (None = NULL). NULL cells' stored values are checked only when
    null_values_checked (a bare SCAN carries its data through untouched)."""
    return {"success": True, "rows": rows, "compare": compare, "keys": keys, "float_tol": float_tol,
            "row_count": len(rows), "null_values_checked": null_values_checked}


def refuse(substring=""):
    return {"success": False, "error_contains": substring}


# ---- projection / filter (test_gpu_executor.cpp:122-452) -------------------------------------------

@case("test_gpu_executor.cpp:122")
def projection_runs_on_gpu():
    n = 50000
    rev = np.array([(i % 997) + 0.5 for i in range(n)])
    plan = make_projection([expr("((double*)out)[idx] = (((const double*)inputs[0])[row]) * 1.18;", ["revenue"],
                                 T.FLOAT64)], make_scan(["revenue"]))
    return plan, [make_column("revenue", T.FLOAT64, rev)], lambda: ok(rows_of(list(rev * 1.18)), "ordered",
                                                                      float_tol=1e-9)


@case("test_gpu_executor.cpp:154")
def filter_compacts_on_gpu():
    ids = [i % 500 for i in range(20000)]
    plan = make_filter([expr("((bool*)out)[idx] = (((const int*)inputs[0])[row]) > 100;", ["id"], T.BOOLEAN)],
                       make_scan(["id"]))
    return plan, [make_column("id", T.INT32, ids)], lambda: ok(rows_of([v for v in ids if v > 100]), "ordered")


@case("test_gpu_executor.cpp:188")
def filter_then_projection_pipeline():
    qty = [i % 10 for i in range(12000)]
    f = make_filter([expr("((bool*)out)[idx] = (((const int*)inputs[0])[row]) > 3;", ["qty"], T.BOOLEAN)],
                    make_scan(["qty"]))
    plan = make_projection([expr("((int*)out)[idx] = (((const int*)inputs[0])[row]) * 2;", ["qty"], T.INT32)], f)
    return plan, [make_column("qty", T.INT32, qty)], lambda: ok(rows_of([v * 2 for v in qty if v > 3]), "ordered")


@case("test_gpu_executor.cpp:227")
def multi_column_filter_gathers_every_column():
    n = 5000
    a = [i % 7 for i in range(n)]
    b = [float(i) for i in range(n)]
    plan = make_filter([expr("((bool*)out)[idx] = (((const int*)inputs[0])[row]) > 4;", ["a"], T.BOOLEAN)],
                       make_scan(["a", "b"]))
    keep = [i for i in range(n) if a[i] > 4]
    return plan, [make_column("a", T.INT32, a), make_column("b", T.FLOAT64, b)], \
        lambda: ok(rows_of([a[i] for i in keep], [b[i] for i in keep]), "ordered")


@case("test_gpu_executor.cpp:265")
def filter_matching_nothing_produces_empty_result():
    plan = make_filter([expr("((bool*)out)[idx] = (((const int*)inputs[0])[row]) > 999;", ["id"], T.BOOLEAN)],
                       make_scan(["id"]))
    return plan, [make_column("id", T.INT32, [1] * 4096)], lambda: ok([], "ordered")


@case("test_gpu_executor.cpp:285")
def nullable_column_passes_through_bare_scan():
    n = 256
    ids = list(range(n))
    valid = [i != 0 for i in range(n)]
    plan = make_scan(["id"])
    return plan, [make_column("id", T.INT32, ids, valid)], \
        lambda: dict(ok(rows_of(ids), "ordered", null_values_checked=True),
                     nulls=[[i, 0] for i in range(n) if not valid[i]])


@case("test_gpu_executor.cpp:322")
def nullable_column_propagates_through_projection():
    n = 128
    v = list(range(n))
    valid = [i not in (3, 100) for i in range(n)]
    plan = make_projection([expr("((int*)out)[idx] = (((const int*)inputs[0])[row]) + 1;", ["v"], T.INT32)],
                           make_scan(["v"]))
    return plan, [make_column("v", T.INT32, v, valid)], \
        lambda: dict(ok(rows_of([v[i] + 1 for i in range(n)]), "ordered"),
                     nulls=[[i, 0] for i in range(n) if not valid[i]])


@case("test_gpu_executor.cpp:370")
def nullable_column_excluded_by_filter_predicate():
    n = 64
    ids = list(range(n))
    v = list(range(n))
    valid = [i != 10 for i in range(n)]
    plan = make_filter([expr("((bool*)out)[idx] = (((const int*)inputs[0])[row]) > 5;", ["v"], T.BOOLEAN)],
                       make_scan(["id", "v"]))
    keep = [i for i in range(n) if i != 10 and v[i] > 5]
    return plan, [make_column("id", T.INT32, ids), make_column("v", T.INT32, v, valid)], \
        lambda: ok(rows_of([ids[i] for i in keep], [v[i] for i in keep]), "ordered")


@case("test_gpu_executor.cpp:410")
def malformed_plan_fails_cleanly():
    plan = make_join("a", "b", ["a"], make_scan([]), make_scan([]))
    plan.children = plan.children[:1]  # a join with one child
    return plan, [], lambda: refuse("")


@case("test_gpu_executor.cpp:421")
def repeated_execution_hits_kernel_cache():
    n = 8192
    v = [float(i) for i in range(n)]
    plan = make_projection([expr("((double*)out)[idx] = (((const double*)inputs[0])[row]) + 7.0;", ["v"],
                                 T.FLOAT64)], make_scan(["v"]))
    return plan, [make_column("v", T.FLOAT64, v)], lambda: ok(rows_of([x + 7.0 for x in v]), "ordered")


# ---- GROUP BY (test_gpu_executor.cpp:455-890, 1338-1440) ---------------------------------------------

@case("test_gpu_executor.cpp:455")
def group_by_sum_on_gpu():
    n = 100000
    k = [i % 1000 for i in range(n)]
    v = [float(i % 64) for i in range(n)]
    plan = make_group_by(["k"], [make_aggregate(A.SUM, "v", T.FLOAT64)], make_scan(["k", "v"]))

    def exp():
        m = defaultdict(float)
        for a, b in zip(k, v):
            m[a] += b
        return ok([[a, m[a]] for a in sorted(m)], "set", keys=1, float_tol=1e-9)
    return plan, [make_column("k", T.INT32, k), make_column("v", T.FLOAT64, v)], exp


@case("test_gpu_executor.cpp:494")
def group_by_count_star_on_gpu():
    n = 60000
    k = [(i * i) % 251 for i in range(n)]
    plan = make_group_by(["k"], [make_aggregate(A.COUNT_STAR, "", T.INT64)], make_scan(["k"]))

    def exp():
        m = defaultdict(int)
        for a in k:
            m[a] += 1
        return ok([[a, m[a]] for a in sorted(m)], "set", keys=1)
    return plan, [make_column("k", T.INT64, k)], exp


@case("test_gpu_executor.cpp:532")
def group_by_min_max_on_gpu():
    n = 50000
    k = [i % 97 for i in range(n)]
    v = [((i * 7919) % 100000) - 50000 for i in range(n)]
    plan = make_group_by(["k"], [make_aggregate(A.MIN, "v", T.INT64), make_aggregate(A.MAX, "v", T.INT64)],
                         make_scan(["k", "v"]))

    def exp():
        m = {}
        for a, b in zip(k, v):
            lo, hi = m.get(a, (b, b))
            m[a] = (min(lo, b), max(hi, b))
        return ok([[a, m[a][0], m[a][1]] for a in sorted(m)], "set", keys=1)
    return plan, [make_column("k", T.INT32, k), make_column("v", T.INT64, v)], exp


@case("test_gpu_executor.cpp:578")
def group_by_multiple_keys_on_gpu():
    n = 80000
    k1 = [(i % 13) - 6 for i in range(n)]
    k2 = [(i % 7) - 3 for i in range(n)]
    v = [float(i % 32) for i in range(n)]
    plan = make_group_by(["k1", "k2"], [make_aggregate(A.SUM, "v", T.FLOAT64)], make_scan(["k1", "k2", "v"]))

    def exp():
        m = defaultdict(float)
        for a, b, c in zip(k1, k2, v):
            m[(a, b)] += c
        return ok([[a, b, m[(a, b)]] for (a, b) in sorted(m)], "set", keys=2, float_tol=1e-9)
    return plan, [make_column("k1", T.INT32, k1), make_column("k2", T.INT64, k2), make_column("v", T.FLOAT64, v)], exp


@case("test_gpu_executor.cpp:622")
def group_by_global_aggregate_on_gpu():
    n = 30000
    v = [float(i % 128) for i in range(n)]
    plan = make_group_by([], [make_aggregate(A.COUNT_STAR, "", T.INT64), make_aggregate(A.SUM, "v", T.FLOAT64)],
                         make_scan(["v"]))
    return plan, [make_column("v", T.FLOAT64, v)], lambda: ok([[n, sum(v)]], "ordered", float_tol=1e-6)


@case("test_gpu_executor.cpp:653")
def group_by_after_filter_on_gpu():
    n = 40000
    k = [i % 50 for i in range(n)]
    v = [i % 30 for i in range(n)]
    f = make_filter([expr("((bool*)out)[idx] = (((const int*)inputs[1])[row]) > 10;", ["k", "v"], T.BOOLEAN)],
                    make_scan(["k", "v"]))
    plan = make_group_by(["k"], [make_aggregate(A.COUNT_STAR, "", T.INT64)], f)

    def exp():
        m = defaultdict(int)
        for a, b in zip(k, v):
            if b > 10:
                m[a] += 1
        return ok([[a, m[a]] for a in sorted(m)], "set", keys=1)
    return plan, [make_column("k", T.INT32, k), make_column("v", T.INT32, v)], exp


@case("test_gpu_executor.cpp:698")
def group_by_sum_of_float_promotes_to_double():
    n = 20000
    k = [i % 4 for i in range(n)]
    v = [float(i % 256) for i in range(n)]
    plan = make_group_by(["k"], [make_aggregate(A.SUM, "v", T.FLOAT64)], make_scan(["k", "v"]))

    def exp():
        m = defaultdict(float)
        for a, b in zip(k, v):
            m[a] += b
        return ok([[a, m[a]] for a in sorted(m)], "set", keys=1, float_tol=1e-6)
    return plan, [make_column("k", T.INT32, k), make_column("v", T.FLOAT32, v)], exp


@case("test_gpu_executor.cpp:733")
def group_by_high_cardinality_on_gpu():
    groups = 200000
    n = groups * 2
    k = [i % groups for i in range(n)]
    v = list(range(n))
    plan = make_group_by(["k"], [make_aggregate(A.COUNT_STAR, "", T.INT64), make_aggregate(A.MAX, "v", T.INT64)],
                         make_scan(["k", "v"]))
    return plan, [make_column("k", T.INT64, k), make_column("v", T.INT64, v)], \
        lambda: ok([[g, 2, g + groups] for g in range(groups)], "set", keys=1)


@case("test_gpu_executor.cpp:772")
def group_by_empty_input_produces_no_groups():
    f = make_filter([expr("((bool*)out)[idx] = (((const int*)inputs[0])[row]) > 999;", ["k"], T.BOOLEAN)],
                    make_scan(["k"]))
    plan = make_group_by(["k"], [make_aggregate(A.COUNT_STAR, "", T.INT64)], f)
    return plan, [make_column("k", T.INT32, [3] * 8192)], lambda: ok([], "set", keys=1)


@case("test_gpu_executor.cpp:797")
def group_by_float_key_refused_cleanly():
    plan = make_group_by(["k"], [make_aggregate(A.COUNT_STAR, "", T.INT64)], make_scan(["k"]))
    return plan, [make_column("k", T.FLOAT64, [1.5] * 1024)], lambda: refuse("integer/boolean")


@case("test_gpu_executor.cpp:812")
def nullable_column_refused_for_group_by_aggregate():
    valid = [i != 0 for i in range(256)]
    plan = make_group_by(["k"], [make_aggregate(A.COUNT_STAR, "", T.INT64)], make_scan(["k"]))
    return plan, [make_column("k", T.INT32, [5] * 256, valid)], lambda: refuse("NULL")


@case("test_gpu_executor.cpp:835")
def group_by_float_min_max_refused_cleanly():
    plan = make_group_by(["k"], [make_aggregate(A.MAX, "v", T.FLOAT64)], make_scan(["k", "v"]))
    return plan, [make_column("k", T.INT32, [1] * 1024), make_column("v", T.FLOAT64, [2.0] * 1024)], \
        lambda: refuse("")


@case("test_gpu_executor.cpp:851")
def group_by_global_aggregate_over_empty_input_refused_cleanly():
    f = make_filter([expr("((bool*)out)[idx] = (((const double*)inputs[0])[row]) > 99.0;", ["v"], T.BOOLEAN)],
                    make_scan(["v"]))
    plan = make_group_by([], [make_aggregate(A.SUM, "v", T.FLOAT64)], f)
    return plan, [make_column("v", T.FLOAT64, [1.0] * 4096)], lambda: refuse("NULL")


@case("test_gpu_executor.cpp:1338")
def group_by_with_projected_smallint_key():
    n = 30000
    k = [i % 7 for i in range(n)]
    p = make_projection([expr("((short*)out)[idx] = ((const short*)inputs[0])[row];", ["k"], T.INT16)],
                        make_scan(["k"]))
    plan = make_group_by(["col0"], [make_aggregate(A.COUNT_STAR, "", T.INT64)], p)

    def exp():
        m = defaultdict(int)
        for a in k:
            m[a] += 1
        return ok([[a, m[a]] for a in sorted(m)], "set", keys=1)
    return plan, [make_column("k", T.INT16, k)], exp


@case("test_gpu_executor.cpp:1387")
def group_by_with_projected_computed_key():
    n = 50000
    k = list(range(n))
    v = [i % 100 for i in range(n)]
    p = make_projection([
        expr("((int*)out)[idx] = (((const int*)inputs[0])[row]) % 10;", ["k"], T.INT32),
        expr("((double*)out)[idx] = (double)(((const int*)inputs[0])[row]);", ["v"], T.FLOAT64),
    ], make_scan(["k", "v"]))
    plan = make_group_by(["col0"], [make_aggregate(A.SUM, "col1", T.FLOAT64)], p)

    def exp():
        m = defaultdict(int)
        for a, b in zip(k, v):
            m[a % 10] += b
        return ok([[a, float(m[a])] for a in sorted(m)], "set", keys=1, float_tol=0.5)
    return plan, [make_column("k", T.INT32, k), make_column("v", T.INT32, v)], exp


# ---- HASH_JOIN (test_gpu_executor.cpp:904-1188) --------------------------------------------------------

def _pairs(a, b):
    return sorted([x, y] for x, y in zip(a, b))


@case("test_gpu_executor.cpp:904")
def inner_join_on_gpu():
    lid = list(range(10000))
    lv = [i * 2 for i in range(10000)]
    rid = list(range(5000))
    rv = [i * 3 for i in range(5000)]
    plan = make_join("lid", "rid", ["lv", "rv"], make_scan(["lid", "lv"]), make_scan(["rid", "rv"]))
    return plan, [make_column("lid", T.INT32, lid), make_column("lv", T.INT32, lv),
                  make_column("rid", T.INT32, rid), make_column("rv", T.INT32, rv)], \
        lambda: ok(sorted([i * 2, i * 3] for i in range(5000)), "multiset")


@case("test_gpu_executor.cpp:943")
def join_many_to_many_on_gpu():
    lid, lv, rid, rv = [], [], [], []
    for k in range(50):
        for i in range(3):
            lid.append(k)
            lv.append(k * 10 + i)
        for j in range(4):
            rid.append(k)
            rv.append(k * 100 + j)
    plan = make_join("lid", "rid", ["lv", "rv"], make_scan(["lid", "lv"]), make_scan(["rid", "rv"]))
    exp = sorted([k * 10 + i, k * 100 + j] for k in range(50) for i in range(3) for j in range(4))
    return plan, [make_column("lid", T.INT32, lid), make_column("lv", T.INT32, lv),
                  make_column("rid", T.INT32, rid), make_column("rv", T.INT32, rv)], lambda: ok(exp, "multiset")


@case("test_gpu_executor.cpp:985")
def join_with_negative_keys_on_gpu():
    n = 2000
    lid = [i - n for i in range(n)]
    lv = list(range(n))
    rv = [i + 1000 for i in range(n)]
    plan = make_join("lid", "rid", ["lv", "rv"], make_scan(["lid", "lv"]), make_scan(["rid", "rv"]))
    return plan, [make_column("lid", T.INT64, lid), make_column("lv", T.INT32, lv),
                  make_column("rid", T.INT64, lid), make_column("rv", T.INT32, rv)], \
        lambda: ok(sorted([i, i + 1000] for i in range(n)), "multiset")


@case("test_gpu_executor.cpp:1019")
def join_output_column_order_is_respected():
    n = 1000
    plan = make_join("lid", "rid", ["rv", "lv"], make_scan(["lid", "lv"]), make_scan(["rid", "rv"]))
    return plan, [make_column("lid", T.INT32, range(n)), make_column("lv", T.INT32, [i + 7 for i in range(n)]),
                  make_column("rid", T.INT32, range(n)), make_column("rv", T.INT32, [i + 9 for i in range(n)])], \
        lambda: ok(sorted([i + 9, i + 7] for i in range(n)), "multiset")


@case("test_gpu_executor.cpp:1055")
def join_after_filter_on_gpu():
    n = 4000
    lv = [i % 100 for i in range(n)]
    f = make_filter([expr("((bool*)out)[idx] = (((const int*)inputs[0])[row]) > 50;", ["lv"], T.BOOLEAN)],
                    make_scan(["lid", "lv"]))
    plan = make_join("lid", "rid", ["lv", "rv"], f, make_scan(["rid", "rv"]))
    exp = sorted([lv[i], i] for i in range(n) if lv[i] > 50)
    return plan, [make_column("lid", T.INT32, range(n)), make_column("lv", T.INT32, lv),
                  make_column("rid", T.INT32, range(n)), make_column("rv", T.INT32, range(n))], \
        lambda: ok(exp, "multiset")


@case("test_gpu_executor.cpp:1094")
def join_matching_nothing_produces_empty_result():
    n = 2048
    plan = make_join("lid", "rid", ["lv", "rv"], make_scan(["lid", "lv"]), make_scan(["rid", "rv"]))
    return plan, [make_column("lid", T.INT32, [1] * n), make_column("lv", T.INT32, [5] * n),
                  make_column("rid", T.INT32, [999] * n), make_column("rv", T.INT32, [7] * n)], \
        lambda: ok([], "multiset")


@case("test_gpu_executor.cpp:1113")
def join_mismatched_key_types_refused_cleanly():
    plan = make_join("lid", "rid", ["lid", "rid"], make_scan(["lid"]), make_scan(["rid"]))
    return plan, [make_column("lid", T.INT32, [3] * 512), make_column("rid", T.INT64, [3] * 512)], \
        lambda: refuse("same type")


@case("test_gpu_executor.cpp:1129")
def join_float_key_refused_cleanly():
    plan = make_join("lid", "rid", ["lid", "rid"], make_scan(["lid"]), make_scan(["rid"]))
    return plan, [make_column("lid", T.FLOAT64, [1.5] * 512), make_column("rid", T.FLOAT64, [1.5] * 512)], \
        lambda: refuse("integer/boolean")


@case("test_gpu_executor.cpp:1142")
def join_ambiguous_output_column_refused_cleanly():
    plan = make_join("id", "id", ["id"], make_scan(["id"]), make_scan(["id"]))
    return plan, [make_column("id", T.INT32, [1] * 512), make_column("id", T.INT32, [1] * 512)], \
        lambda: refuse("ambiguous")


@case("test_gpu_executor.cpp:1156")
def join_composite_key_refused_cleanly():
    plan = make_join("l1", "r1", ["l1"], make_scan(["l1"]), make_scan(["r1"]))
    plan.build_keys.append("l1")
    plan.probe_keys.append("r1")
    return plan, [make_column("l1", T.INT32, [1] * 512), make_column("r1", T.INT32, [1] * 512)], \
        lambda: refuse("exactly one equality key")


# ---- CROSS_PRODUCT (test_gpu_executor.cpp:1191-1336) ---------------------------------------------------

@case("test_gpu_executor.cpp:1191")
def cross_product_on_gpu():
    plan = make_cross_product(["lv", "rv"], make_scan(["lv"]), make_scan(["rv"]))
    return plan, [make_column("lv", T.INT32, [10, 20, 30]), make_column("rv", T.INT32, [1, 2, 3, 4])], \
        lambda: ok(rows_of([10] * 4 + [20] * 4 + [30] * 4, [1, 2, 3, 4] * 3), "ordered")


@case("test_gpu_executor.cpp:1215")
def cross_product_mixed_widths_and_column_order():
    plan = make_cross_product(["rk", "lval", "lk"], make_scan(["lk", "lval"]), make_scan(["rk"]))
    return plan, [make_column("lk", T.INT32, [7, 8]), make_column("lval", T.FLOAT64, [1.5, 2.5]),
                  make_column("rk", T.INT64, [100, 200, 300])], \
        lambda: ok(rows_of([100, 200, 300] * 2, [1.5] * 3 + [2.5] * 3, [7] * 3 + [8] * 3), "ordered")


@case("test_gpu_executor.cpp:1240")
def projection_over_cross_product_on_gpu():
    lval = [i * 0.25 for i in range(500)]
    rval = [j * 0.5 + 1.0 for j in range(400)]
    cross = make_cross_product(["lval", "rval"], make_scan(["lval"]), make_scan(["rval"]))
    plan = make_projection([expr("((double*)out)[idx] = (((const double*)inputs[0])[row]) * "
                                 "(((const double*)inputs[1])[row]);", ["lval", "rval"], T.FLOAT64)], cross)
    return plan, [make_column("lval", T.FLOAT64, lval), make_column("rval", T.FLOAT64, rval)], \
        lambda: ok(rows_of([a * b for a in lval for b in rval]), "ordered", float_tol=1e-9)


@case("test_gpu_executor.cpp:1281")
def cross_product_empty_side_produces_no_rows():
    plan = make_cross_product(["lv", "rv"], make_scan(["lv"]), make_scan(["rv"]))
    return plan, [make_column("lv", T.INT32, [1, 2, 3]), make_column("rv", T.INT32, [])], lambda: ok([], "ordered")


@case("test_gpu_executor.cpp:1302")
def cross_product_oversize_refused_cleanly():
    n = 70000
    plan = make_cross_product(["lv", "rv"], make_scan(["lv"]), make_scan(["rv"]))
    return plan, [make_column("lv", T.INT32, [1] * n), make_column("rv", T.INT32, [2] * n)], lambda: refuse("too large")


@case("test_gpu_executor.cpp:1318")
def cross_product_ambiguous_output_column_refused_cleanly():
    plan = make_cross_product(["id"], make_scan(["id"]), make_scan(["id"]))
    return plan, [make_column("id", T.INT32, [1, 2]), make_column("id", T.INT32, [3, 4])], lambda: refuse("ambiguous")


# ---- the legacy filter primitive's edge cases (cuda_engine/tests/test_gpu_filter.cu:59-145) ---------
# FilterGreaterThanInt32 is a stand-alone x > t compaction; here it is the FILTER operator.

def _gt_filter(values, threshold):
    plan = make_filter([expr(f"((bool*)out)[idx] = (((const int*)inputs[0])[row]) > {threshold};", ["x"],
                             T.BOOLEAN)], make_scan(["x"]))
    return plan, [make_column("x", T.INT32, values)], \
        lambda: ok(rows_of([v for v in values if v > threshold]), "ordered")


@case("test_gpu_filter.cu:59")
def filter_gt_empty_input():
    return _gt_filter([], 0)


@case("test_gpu_filter.cu:66")
def filter_gt_all_pass():
    return _gt_filter([1, 2, 3, 4], 0)


@case("test_gpu_filter.cu:105")
def filter_gt_boundary_not_strictly_greater():
    return _gt_filter([5, 5, 5], 5)


@case("test_gpu_filter.cu:128")
def filter_gt_negative_threshold():
    return _gt_filter([-10, -5, 0, 5, -1], -5)


@case("test_gpu_filter.cu:136")
def filter_gt_int32_extremes():
    return _gt_filter([-2147483648, 2147483647, 0, -1], 2147483646)


@case("test_gpu_filter.cu:113")
def filter_gt_large_array():
    vals = [((i * 2654435761) % 2000003) - 1000000 for i in range(300000)]
    return _gt_filter(vals, 12345)
