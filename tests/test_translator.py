"""Bound expression -> engine expression (vectisdb_b200.translate over vgpu_translate_expression),
following the reference extension's translator (extension/src/expression_translator.cpp:287-493):
the benchmark queries' expressions translate to exactly the statements their plans carry, the literal
and operator forms match the reference's, refusals carry its reasons, and a translated plan computes
what the plan oracle computes."""
import numpy as np
import pytest

from vectisdb_b200 import abi, make_aggregate, make_column, make_filter, make_group_by, make_projection, make_scan
from vectisdb_b200 import workloads as W
from vectisdb_b200.engine import GpuAggregateKind as A, GpuValueType as T, generate_source, nvrtc_compile_check
from vectisdb_b200.translate import FP32, STRICT_FP, cast, cmp, col, const, fn, translate


def _stmt(e, flags=0):
    return translate(e, flags).generated_cuda_source


def test_benchmark_expressions_translate_to_the_plans_statements():
    c0 = W.c0_plan(0.5, 7)
    proj, filt = c0.children[0], c0.children[0].children[0]
    got = [translate(cmp("<", col("v", T.FLOAT64), const(0.5, T.FLOAT64))),
           translate(cmp("!=", fn("%", T.INT64, col("w", T.INT64), const(7, T.INT64)), const(0, T.INT64))),
           translate(col("k", T.INT32)),
           translate(fn("+", T.FLOAT64, fn("*", T.FLOAT64, col("v", T.FLOAT64), const(2, T.FLOAT64)),
                        const(1, T.FLOAT64))),
           translate(col("w", T.INT64))]
    want = list(filt.expressions) + list(proj.expressions)
    for g, w in zip(got, want):
        assert g.generated_cuda_source == w.generated_cuda_source
        assert g.input_columns == w.input_columns and g.output_type == w.output_type
    ts = translate(cmp(">", col("ts", T.INT64), const(12345, T.INT64)))
    assert ts.generated_cuda_source == W.c1_plan(12345).children[0].expressions[0].generated_cuda_source


def test_literal_forms():
    assert _stmt(const(2.0, T.FLOAT32)) == "((float*)out)[idx] = 2.0f;"  # a decimal point before the suffix
    assert _stmt(const(0.1, T.FLOAT64)) == "((double*)out)[idx] = 0.10000000000000001;"
    assert _stmt(const(-3, T.INT32)) == "((int*)out)[idx] = -3;"
    assert _stmt(const(1 << 40, T.INT64)) == "((long long*)out)[idx] = 1099511627776LL;"
    assert _stmt(const(1, T.BOOLEAN)) == "((bool*)out)[idx] = true;"
    assert _stmt(const(7, T.INT16)) == "((short*)out)[idx] = 7;"


def test_columns_share_slots_in_first_reference_order():
    e = fn("+", T.INT64, fn("*", T.INT64, col("b", T.INT64), col("a", T.INT64)), col("b", T.INT64))
    t = translate(e)
    assert t.input_columns == ["b", "a"]
    assert t.generated_cuda_source == ("((long long*)out)[idx] = ((((const long long*)inputs[0])[row] * "
                                       "((const long long*)inputs[1])[row]) + ((const long long*)inputs[0])[row]);")


def test_operators_functions_and_casts():
    x, i = col("x", T.FLOAT64), col("i", T.INT32)
    assert _stmt(fn("-", T.FLOAT64, x)) == "((double*)out)[idx] = (-((const double*)inputs[0])[row]);"
    assert _stmt(fn("%", T.FLOAT64, x, const(2.5, T.FLOAT64))) == \
        "((double*)out)[idx] = fmod((double)(((const double*)inputs[0])[row]), (double)(2.5));"
    assert _stmt(fn("ln", T.FLOAT64, x)) == "((double*)out)[idx] = log((double)(((const double*)inputs[0])[row]));"
    assert _stmt(fn("log", T.FLOAT64, x)).startswith("((double*)out)[idx] = log10(")  # DuckDB log is base 10
    assert _stmt(fn("ceiling", T.FLOAT64, x)).startswith("((double*)out)[idx] = ceil(")
    assert _stmt(fn("pow", T.FLOAT64, x, const(2.0, T.FLOAT64))).startswith("((double*)out)[idx] = pow(")
    assert _stmt(fn("abs", T.INT32, i)) == ("((int*)out)[idx] = ((((const int*)inputs[0])[row]) < 0 ? "
                                            "-(((const int*)inputs[0])[row]) : (((const int*)inputs[0])[row]));")
    assert _stmt(fn("abs", T.FLOAT64, x)) == "((double*)out)[idx] = fabs((double)(((const double*)inputs[0])[row]));"
    assert _stmt(cast(i, T.INT64)) == "((long long*)out)[idx] = ((long long)(((const int*)inputs[0])[row]));"
    assert _stmt(cast(i, T.INT32)) == "((int*)out)[idx] = ((const int*)inputs[0])[row];"
    assert _stmt(fn("sin", T.FLOAT64, x), FP32) == \
        "((double*)out)[idx] = (double)(sinf((float)(((const double*)inputs[0])[row])));"
    assert _stmt(fn("sqrt", T.FLOAT64, x), STRICT_FP).startswith("((double*)out)[idx] = sqrt(")
    assert _stmt(cmp("<>", i, const(3, T.INT32))) == "((bool*)out)[idx] = (((const int*)inputs[0])[row] != 3);"


@pytest.mark.parametrize("expr,reason", [
    (lambda: cast(col("w", T.INT64), T.INT32), "does not agree"),            # narrowing: DuckDB raises
    (lambda: cast(col("x", T.FLOAT64), T.INT64), "does not agree"),          # float -> integer rounds
    (lambda: cast(col("x", T.FLOAT64), T.FLOAT32), "does not agree"),        # DuckDB range-checks
    (lambda: const(None, T.INT32), "NULL constants"),
    (lambda: const(float("inf"), T.FLOAT64), "non-finite"),
    (lambda: fn("sqrt", T.FLOAT32, col("f", T.FLOAT32)), "returns DOUBLE"),
    (lambda: fn("regexp_matches", T.BOOLEAN, col("x", T.FLOAT64)), "unsupported function"),
    (lambda: cmp("LIKE", col("x", T.FLOAT64), const(1.0, T.FLOAT64)), "unsupported comparison"),
    (lambda: fn("+", T.HUGEINT, col("h", T.HUGEINT), col("h", T.HUGEINT)), "HUGEINT"),
])
def test_refusals_carry_the_reason(expr, reason):
    with pytest.raises(abi.VgpuError) as e:
        translate(expr())
    assert e.value.status == abi.ERR_UNSUPPORTED and reason in str(e.value)


def test_strict_fp_refuses_transcendentals():
    with pytest.raises(abi.VgpuError) as e:
        translate(fn("exp", T.FLOAT64, col("x", T.FLOAT64)), STRICT_FP)
    assert "bit-identical" in str(e.value)


def test_translated_plan_matches_the_plan_oracle_and_compiles():
    """SELECT k, SUM(sqrt(v) * 3 - w), COUNT(*) WHERE v >= 0.25 AND k % 3 = 1 GROUP BY k, built from
    bound expressions: its fused kernels compile and the plan oracle evaluates it like numpy."""
    from oracle.plan_oracle import evaluate
    wl = W.c0(n=20_000)
    k, v, w = [c.data for c in wl.inputs]
    filt = make_filter([translate(cmp(">=", col("v", T.FLOAT64), const(0.25, T.FLOAT64))),
                        translate(cmp("=", fn("%", T.INT32, col("k", T.INT32), const(3, T.INT32)),
                                      const(1, T.INT32)))], make_scan(["k", "v", "w"]))
    proj = make_projection([translate(col("k", T.INT32)),
                            translate(fn("-", T.FLOAT64, fn("*", T.FLOAT64, fn("sqrt", T.FLOAT64, col("v", T.FLOAT64)),
                                                            const(3, T.FLOAT64)),
                                         cast(col("w", T.INT64), T.FLOAT64)))], filt)
    plan = make_group_by(["col0"], [make_aggregate(A.SUM, "col1", T.FLOAT64), make_aggregate(A.COUNT_STAR, "", T.INT64)],
                         proj)
    for tu in generate_source(plan, wl.inputs).split("//@@VGPU_TU@@"):
        assert nvrtc_compile_check(tu) > 1000
    keys, sums, counts = [np.asarray(c.data) for c in evaluate(plan, wl.inputs)]
    m = (v >= 0.25) & (k % 3 == 1)
    exp_keys = np.unique(k[m])
    assert np.array_equal(np.sort(keys), exp_keys)
    order = np.argsort(keys)
    x = np.sqrt(v[m]) * 3.0 - w[m].astype(np.float64)
    exp_sums = np.array([x[k[m] == kk].sum() for kk in exp_keys])
    assert np.allclose(sums[order], exp_sums, rtol=1e-12, atol=1e-9)
    assert np.array_equal(counts[order], np.array([(k[m] == kk).sum() for kk in exp_keys]))


@pytest.mark.gpu
def test_translated_plan_on_the_gpu_matches_the_plan_oracle():
    from oracle.plan_oracle import evaluate
    from vectisdb_b200 import GpuEngine
    wl = W.c0(n=300_000)
    filt = make_filter([translate(cmp(">=", col("v", T.FLOAT64), const(0.25, T.FLOAT64))),
                        translate(cmp("=", fn("%", T.INT32, col("k", T.INT32), const(3, T.INT32)),
                                      const(1, T.INT32)))], make_scan(["k", "v", "w"]))
    proj = make_projection([translate(col("k", T.INT32)),
                            translate(fn("-", T.FLOAT64, fn("*", T.FLOAT64, fn("sqrt", T.FLOAT64, col("v", T.FLOAT64)),
                                                            const(3, T.FLOAT64)),
                                         cast(col("w", T.INT64), T.FLOAT64)))], filt)
    plan = make_group_by(["col0"], [make_aggregate(A.SUM, "col1", T.FLOAT64), make_aggregate(A.COUNT_STAR, "", T.INT64)],
                         proj)
    r = GpuEngine.instance().execute_plan(plan, wl.inputs)
    assert r.success, r.error_message
    got = [np.asarray(c.data) for c in r.columns]
    exp = [np.asarray(c.data) for c in evaluate(plan, wl.inputs)]
    og, oe = np.argsort(got[0]), np.argsort(exp[0])
    assert np.array_equal(got[0][og], exp[0][oe]) and np.array_equal(got[2][og], exp[2][oe])
    assert np.all(np.abs(got[1][og] - exp[1][oe]) <= 1e-12 * np.abs(exp[1][oe]))
