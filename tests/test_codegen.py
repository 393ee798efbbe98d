"""Per-query code generation: the fused kernels for every benchmark query and every reference test
plan compile with NVRTC for sm_100a on a machine without a GPU; malformed expressions are refused."""
import pytest

from vectisdb_b200 import abi
from vectisdb_b200 import workloads as W
from vectisdb_b200.engine import (GpuValueType as T, generate_source, make_column, make_expr, make_filter,
                                  make_scan, nvrtc_compile_check)
from reference_cases import CASES


def _compile_all(src):
    sizes = []
    for tu in src.split("//@@VGPU_TU@@"):
        sizes.append(nvrtc_compile_check(tu))
    return sizes


@pytest.mark.parametrize("name", ["c0", "c1"])
def test_benchmark_query_kernels_compile(name):
    wl = W.c0(n=64) if name == "c0" else W.c1(n=64)
    src = generate_source(wl.plan, wl.inputs)
    assert "vgpu_gb_direct" in src and "vgpu_gb_bucket" in src and "vgpu_gb_dbucket" in src
    assert "vgpu_gb_sample" in src and "vgpu_hmap" in src
    assert "stage_copy(" in src and "stage_wait(" in src
    assert all(s > 1000 for s in _compile_all(src))


def test_filter_materialize_kernel_compiles_and_fuses():
    wl = W.c0(n=64)
    plan = wl.plan.children[0].children[0]  # the FILTER over the SCAN
    src = generate_source(plan, wl.inputs)
    assert "vgpu_mat_count" in src and "vgpu_mat_write" in src
    # both predicates evaluate in registers: no reference-style inputs[] access survives
    assert "inputs[" not in src
    _compile_all(src)


@pytest.mark.parametrize("name", [n for n in sorted(CASES) if "refused" not in n and "malformed" not in n])
def test_reference_plans_compile(name):
    _, build = CASES[name]
    plan, inputs, _ = build()
    try:
        src = generate_source(plan, inputs)
    except abi.VgpuError as e:  # joins / cross products need device-side sizes; covered on the GPU
        assert e.status == abi.ERR_UNSUPPORTED
        return
    _compile_all(src)


def test_expression_outside_the_reference_forms_is_refused():
    bad = make_filter([make_expr("((bool*)out)[idx] = inputs[0] != 0;", ["k"], T.BOOLEAN)], make_scan(["k"]))
    with pytest.raises(abi.VgpuError) as e:
        generate_source(bad, [make_column("k", T.INT32, [1, 2])])
    assert e.value.status == abi.ERR_UNSUPPORTED


def test_width_mismatch_is_refused():
    bad = make_filter([make_expr("((bool*)out)[idx] = ((const long long*)inputs[0])[row] > 1;", ["k"], T.BOOLEAN)],
                      make_scan(["k"]))
    with pytest.raises(abi.VgpuError) as e:
        generate_source(bad, [make_column("k", T.INT32, [1, 2])])
    assert e.value.status == abi.ERR_UNSUPPORTED


def test_nvrtc_reports_compile_errors():
    with pytest.raises(abi.VgpuError) as e:
        nvrtc_compile_check('extern "C" __global__ void k() { this is not cuda; }')
    assert e.value.status == abi.ERR_COMPILE


def test_engine_nvrtc_is_independent_of_an_older_preloaded_copy():
    """A process that already holds another NVRTC of the same soname (PyTorch's wheel ships one) must
    not lend it to the engine: the generated kernels use sm_100 instruction forms that only the
    engine's own toolkit NVRTC assembles. Runs in a child process so the preload stays contained."""
    import os
    import subprocess
    import sys
    torch = pytest.importorskip("torch")
    lib = os.path.join(os.path.dirname(torch.__file__), "..", "nvidia", "cuda_nvrtc", "lib", "libnvrtc.so.12")
    if not os.path.exists(lib):
        pytest.skip("no separately packaged NVRTC to preload")
    code = (
        "import ctypes, sys\n"
        f"ctypes.CDLL({lib!r}, mode=ctypes.RTLD_GLOBAL)\n"
        "from vectisdb_b200 import workloads as W\n"
        "from vectisdb_b200.engine import generate_source, nvrtc_compile_check\n"
        "src = generate_source(W.c1(n=64).plan, W.c1(n=64).inputs)\n"
        "print(min(nvrtc_compile_check(tu) for tu in src.split('//@@VGPU_TU@@')))\n")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    assert int(out.stdout.strip().splitlines()[-1]) > 1000


def test_stream_pipeline_supports_projection_chains_only():
    """GpuStreamPipeline::Supports: PROJECTION+ over a SCAN with resolvable inputs; no filter."""
    from vectisdb_b200 import StreamPipeline, make_projection
    scan = make_scan(["a", "b"])
    ok = make_projection([make_expr("((long long*)out)[idx] = ((const long long*)inputs[0])[row] + 1;", ["a"],
                                    T.INT64)], scan)
    assert StreamPipeline.supports(ok)
    assert StreamPipeline.supports(make_projection(
        [make_expr("((long long*)out)[idx] = ((const long long*)inputs[0])[row];", ["col0"], T.INT64)], ok))
    bad_input = make_projection([make_expr("((long long*)out)[idx] = ((const long long*)inputs[0])[row];", ["zz"],
                                           T.INT64)], scan)
    assert not StreamPipeline.supports(bad_input)
    filt = make_filter([make_expr("((bool*)out)[idx] = ((const long long*)inputs[0])[row] > 0;", ["a"], T.BOOLEAN)],
                       scan)
    assert not StreamPipeline.supports(filt)
    assert not StreamPipeline.supports(scan)


def test_join_source_kernels_compile_single_and_multi_match():
    """The join + group-by query's fused kernels, for a unique-key right side, for repeated keys (each
    probe row expands into its run of matches) and for repeated keys whose right column sits inline in
    the dense table (one slot per match): materialization, key statistics and the one-pass group-by all
    compile; right columns are never read at left row positions."""
    wl = W.c2(probe_n=64, build_n=16, miss_lo=16, miss_span=16)
    src = generate_source(wl.plan, wl.inputs)
    tus = src.split("//@@VGPU_TU@@")
    # materialize: unique, run, inline-run; key statistics: run; group-by: unique, run, inline-run
    assert len(tus) == 7
    assert "vgpu_join_find" in tus[0] and "vgpu_join_run" in tus[1] and "vgpu_join_run" in tus[5]
    assert "vgpu_join_minline(" in tus[3] and "vgpu_join_minline(" in tus[6]
    assert "vgpu_join_minline_value(je[r], jx_" in tus[6]
    assert "for (u32 jx_ = 0; jx_ < jn_; ++jx_)" in tus[5] and "for (u32 jx_ = 0; jx_ < jn_; ++jx_)" in tus[6]
    # the right column g (source 0) is loaded only through the lookup, never by load_rows at row0
    for t in tus[4:]:
        assert "load_rows<int, 8>((const int*)a.w[2]" not in t
    assert all(s > 1000 for s in _compile_all(src))


def _min_per_column_plan(m):
    """GROUP BY k with MIN over each of m INT64 columns: every MIN adds a state word and an output word."""
    import numpy as np
    from vectisdb_b200.engine import GpuAggregateKind as A, GpuTableRef, make_aggregate, make_group_by
    cols = [make_column("k", T.INT32, np.arange(64, dtype=np.int32))]
    cols += [make_column(f"x{i}", T.INT64, np.arange(64, dtype=np.int64)) for i in range(m)]
    plan = make_group_by(["k"], [make_aggregate(A.MIN, f"x{i}", T.INT64) for i in range(m)],
                         make_scan([c.name for c in cols], GpuTableRef("memory", "main", "wide")))
    return plan, cols


def test_one_pass_group_by_compacts_in_its_last_cta_while_argument_words_allow():
    """The one-pass group-by's compaction runs in the CTA that finishes its merge last (a ticket the init
    kernel zeroes), with no separate final kernel -- unless the ticket's argument word would reach the
    reserved key words: then the single-CTA final kernel runs as its own launch. Both forms compile."""
    wl = W.c0(n=4096)
    src = generate_source(wl.plan, wl.inputs)
    assert "vgpu_last" in src and "vgpu_gb_direct_final" not in src
    for m, fused in ((21, True), (22, False)):
        plan, cols = _min_per_column_plan(m)
        src = generate_source(plan, cols)
        assert ("vgpu_last" in src) == fused and ("vgpu_gb_direct_final" in src) == (not fused), m
        assert all(s > 1000 for s in _compile_all(src))


def test_filtered_materialization_stages_kept_rows_for_coalesced_writes():
    """A filter + projection writes each tile's kept rows from shared memory as one run per column, the
    NULL masks included when an output is nullable."""
    wl = W.cp(n=4096)
    src = generate_source(wl.plan, wl.inputs)
    write = src[src.index("vgpu_mat_write("):]
    assert "vgpu_st0[rank] = o0[r];" in write and "[base + i] = vgpu_st0[i];" in write
    plan, inputs, _ = CASES["nullable_column_excluded_by_filter_predicate"][1]()
    src = generate_source(plan, inputs)
    assert "vgpu_sv" in src[src.index("vgpu_mat_write("):]
