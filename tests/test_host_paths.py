"""Host-side paths that need no GPU: the Python binding's reuse of serialized plans, and the bench's
clock sampler on a machine without a GPU."""
import importlib.util
from pathlib import Path

from vectisdb_b200 import workloads as W
from vectisdb_b200.engine import _PLAN_MEMO, serialize_plan_memo


def test_plan_memo_reuses_unchanged_plans_and_rebuilds_changed_ones():
    wl = W.c0(n=1024)
    first, keep1 = serialize_plan_memo(wl.plan)
    again, keep2 = serialize_plan_memo(wl.plan)
    assert again is first and keep2 is keep1  # unchanged plan: the same serialized form
    expr = wl.plan.children[0].expressions[1]  # the projection's v * 2.0 + 1.0
    expr.generated_cuda_source = expr.generated_cuda_source.replace("2.0", "3.0")
    changed, _ = serialize_plan_memo(wl.plan)
    assert changed is not first
    assert b"3.0" in changed.nodes[1].expressions[1].source
    wl.plan.aggregates[0].input_column = wl.plan.aggregates[0].input_column  # same value: still reused
    assert serialize_plan_memo(wl.plan)[0] is changed


def test_plan_memo_is_bounded():
    plans = [W.c0(n=64).plan for _ in range(300)]
    for p in plans:
        serialize_plan_memo(p)
    assert len(_PLAN_MEMO) <= 256


def test_clock_sampler_reports_unavailable_without_a_gpu():
    spec = importlib.util.spec_from_file_location("bench_mod", Path(__file__).resolve().parents[1] / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    s = bench.ClockSampler(0)
    s.start()
    s.mark_begin()
    s.mark_end()
    out = s.stop()
    assert set(out) >= {"sm_mhz", "sm_max_mhz", "reasons"}


def test_reference_arm_prints_one_contract_line():
    """bench.py --impl reference runs the CPU restatement (no GPU needed) and prints one JSON line with
    the keys the bench contract requires, its cpu_baseline and e2e describing the same run."""
    import json
    import subprocess
    import sys
    root = Path(__file__).resolve().parents[1]
    r = subprocess.run([sys.executable, str(root / "bench.py"), "--impl", "reference", "--config", "c0", "--steps", "1",
                        "--warmup", "1"], capture_output=True, text=True, timeout=600, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["steps"] == 1 and line["value"] > 0
    cpu = line["cpu_baseline"]
    assert cpu["value"] == line["value"] and cpu["kind"] == "port" and cpu["cores"] >= 1 and "not DuckDB" in cpu["label"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun the reference arm's other ranks exit 0 at once, printing nothing."""
    import os
    import subprocess
    import sys
    root = Path(__file__).resolve().parents[1]
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    r = subprocess.run([sys.executable, str(root / "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
                        "--warmup", "1"], capture_output=True, text=True, timeout=300, cwd=root, env=env)
    assert r.returncode == 0 and r.stdout.strip() == "", (r.stdout[-500:], r.stderr[-500:])
