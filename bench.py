"""Benchmark of the GPU execution path (the DuckDB hot path: fused filter/projection, GROUP BY, join,
cross product, batching, serving) on the benchmark queries. The headline is the high-cardinality
group-by (c1):

    SELECT a, b, SUM(amt), AVG(v), COUNT(*), MAX(ts) FROM t WHERE ts > median(ts) GROUP BY a, b
    2^27 rows: a INT32 Zipf(1.1) over 2^20, b INT32 U[0,16), amt DECIMAL(18,2) cents, v DOUBLE, ts BIGINT

    python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference] [--config c1|c0|cp|c2|c2dup|c2b|c3|c4]

One step = one execution of the query over the whole table. `value` is rows/s with the base columns
resident in the device column cache (the timed region starts with inputs in HBM, results stay on
the device); `e2e` is the same query through the public API from pinned host buffers, host-to-device
copies and the device-to-host read of the result inside every step. The result of the last timed step
is compared with the oracle (outside the timed region) and `parity` says whether it matched. With
the c1 headline on one GPU, `per_config` adds every other query of the benchmark measured the same way
(c0 filter + group-by, cp filter + projection, c2 join + group-by, c2dup the join with repeated build
keys, c2b filtered cross product, c3 batched vs plain, c4 served vs serial with p50/p99).
Multi-GPU runs (torchrun) are replicas: every rank runs the full query on its own table (weak scaling),
timed as the max over ranks. `--impl reference` times the CPU restatement of the query (DuckDB is not
installed in this image) on all host cores, on the same full-size table.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PEAKS = ROOT / "MEASURED_PEAKS.json"
CPU_BASELINE_LABEL = "C++ restatement of the query (OpenMP, oracle/oracle.cpp), not DuckDB: DuckDB is not installed"
PLAIN_CONFIGS = ("c0", "c1", "c2", "c2b", "cp", "c2dup")
PER_CONFIG_ORDER = ("c0", "cp", "c2", "c2dup", "c2b", "c3", "c4", "c1_sharded")


def hbm_peak():
    if PEAKS.exists():
        return float(json.loads(PEAKS.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clocks, power and clock-event (throttle) reasons of one GPU, sampled every 50 ms by a thread
    of this process through NVML -- the library nvidia-smi reports from -- so no second process competes
    with the timed region for the driver. mark_begin()/mark_end() bracket the timed region; the summary
    covers the samples inside it (or the two nearest when it is shorter than a sampling period).
    Falls back to an `nvidia-smi -lms` subprocess when NVML bindings are missing."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASON_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
                   "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80}

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.thread = None
        self.samples = []  # (time, sm MHz, max sm MHz, power W, reason bits)
        self.window = [None, None]
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"vgpu_clocks_{os.getpid()}.csv"

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:  # the CUDA device's own PCI address: NVML numbers GPUs without CUDA_VISIBLE_DEVICES
            import torch
            pr = torch.cuda.get_device_properties(torch.cuda.current_device())
            bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.gpu)

    def start(self):
        try:
            nv, h = self._nvml_handle()
        except Exception:
            return self._start_smi()
        import threading
        self.stop_flag = threading.Event()

        def run():
            while not self.stop_flag.is_set():
                try:
                    self.samples.append((time.perf_counter(), nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM),
                                         nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM),
                                         nv.nvmlDeviceGetPowerUsage(h) / 1000.0,
                                         nv.nvmlDeviceGetCurrentClocksEventReasons(h)))
                except Exception:
                    pass
                self.stop_flag.wait(0.05)

        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()
        time.sleep(0.12)

    def mark_begin(self):
        self.window[0] = time.perf_counter()

    def mark_end(self):
        self.window[1] = time.perf_counter()

    def _start_smi(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
            return
        # nvidia-smi's start-up (NVML initialisation) competes with the driver for a moment: wait for
        # its first sample (callers also keep the first second after this untimed).
        deadline = time.time() + 5.0
        while time.time() < deadline and self.proc.poll() is None:
            if self.path.exists() and self.path.read_text().count("\n") >= 1:
                break
            time.sleep(0.02)
        time.sleep(0.1)

    def stop(self) -> dict:
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join()
            rows = self.samples
            t0, t1 = self.window
            if t0 is not None and t1 is not None:
                inside = [r for r in rows if t0 <= r[0] <= t1]
                if len(inside) < 2:  # a region shorter than the period: the samples around it
                    inside = sorted(rows, key=lambda r: min(abs(r[0] - t0), abs(r[0] - t1)))[:2]
                rows = inside
            if not rows:
                return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "source": "nvml"}
            reasons = sorted({k for r in rows for k, bit in self.REASON_BITS.items() if r[4] & bit})
            return {"sm_mhz": float(np.median([r[1] for r in rows])), "sm_max_mhz": float(max(r[2] for r in rows)),
                    "power_w": float(np.median([r[3] for r in rows])), "reasons": reasons, "samples": len(rows),
                    "source": "nvml"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        rows = [r.split(", ") for r in self.path.read_text().strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if "Active" == r[5 + i].strip()})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "source": "nvidia-smi"}


def max_over_ranks(value: float, world: int, device: str = "cuda") -> float:
    """The largest of every rank's `value` (a timed region's milliseconds): the job is as slow as its
    slowest replica. Every rank calls it, in the same order."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ---- workloads, oracle checks, algorithmic bytes ----------------------------------------------------

def make_workload(name: str, pinned: bool, rows: int = 0):
    """The named benchmark query on its full-size table, or on `rows` rows (probe rows for c2/c2dup,
    side length for c2b) for small profiling cases."""
    from vectisdb_b200 import workloads as W
    make = {"c0": W.c0, "c1": W.c1, "cp": W.cp}
    if name in make:
        return make[name](n=rows, pinned=pinned) if rows else make[name](pinned=pinned)
    if name in ("c2", "c2dup"):
        fn = W.c2 if name == "c2" else W.c2dup
        return fn(probe_n=rows, pinned=pinned) if rows else fn(pinned=pinned)
    return W.c2b(side=rows) if rows else W.c2b()


def oracle_result(name: str, wl):
    """The oracle's answer for the workload (the checker, and the timed CPU baseline's work)."""
    from oracle import oracle as O
    cols = [c.data for c in wl.inputs]
    if name == "c0":
        return O.c0(*cols, wl.params["v_lt"], wl.params["w_mod"])
    if name == "cp":
        return O.cp(*cols, 0.5, 7)
    if name == "c1":
        return O.c1(*cols, wl.params["ts_gt"])
    if name in ("c2", "c2dup"):
        pkey, x, bkey, g = cols
        return O.c2(bkey, g, pkey, x)
    a, b = cols
    return O.c2b(a, b, wl.params["modulus"])


def _close(got, exp, rel=1e-12):
    got, exp = np.asarray(got, np.float64), np.asarray(exp, np.float64)
    return bool(got.shape == exp.shape and np.all(np.abs(got - exp) <= rel * np.maximum(np.abs(exp), 1e-300)))


def parity_check(name: str, cols: list, exp) -> bool:
    """Engine result columns (host arrays, engine order) against the oracle: keys, counts, MIN/MAX,
    DECIMAL sums and projected/joined values bit-exact; DOUBLE sums and averages within 1e-12 relative."""
    eq = np.array_equal
    if name == "c0":
        k, s, c, mn, mx = cols
        o = np.argsort(k)
        return eq(k[o], exp["k"]) and eq(c[o], exp["count"]) and eq(mn[o], exp["min"]) and \
            eq(mx[o], exp["max"]) and _close(s[o], exp["sum"])
    if name == "cp":
        return all(eq(c, exp[key]) for c, key in zip(cols, ("k", "v", "w")))
    if name == "c1":
        a, b, s, avg, c, mx = cols
        o = np.lexsort((b, a))
        return len(a) == len(exp["a"]) and eq(a[o], exp["a"]) and eq(b[o], exp["b"]) and \
            eq(c[o], exp["count"]) and eq(mx[o], exp["max"]) and eq(s[o]["lower"], exp["sum_lo"]) and \
            eq(s[o]["upper"], exp["sum_hi"]) and _close(avg[o], exp["avg"])
    if name in ("c2", "c2dup"):
        g, s = cols
        o = np.argsort(g)
        return eq(g[o], exp["g"]) and _close(s[o], exp["sum"])
    count, ea, eb = exp
    return len(cols[0]) == count and eq(cols[0], ea) and eq(cols[1], eb)


# Kernels whose algorithmic bytes the engine reports per launch once it knows them: the partition
# scatter (columns read once + the records it wrote -- fewer than the passing rows when heavy keys are
# pre-aggregated) and the direct-partitioned bucket pass (those records read once + the groups written).
ENGINE_COUNTED = ("vgpu_gb_part_scatter", "vgpu_gb_dbucket")


def algorithmic_bytes(name: str, wl, kernel: str, passing: int, groups: int) -> int:
    """Bytes a kernel must move per launch by its role (inputs read once, outputs written once)."""
    n = wl.rows
    if name == "c1":
        return {"vgpu_gb_part_count": 16 * n,                     # a, b, ts
                "vgpu_gb_part_scatter": 32 * n + 32 * passing,    # all columns in; key+3 values out
                "vgpu_gb_bucket": 32 * passing + 48 * groups,     # partitioned rows in; groups out
                "vgpu_gb_dbucket": 32 * passing + 48 * groups,    # partitioned rows in; groups out
                }.get(kernel, 0)
    if name == "c0":
        return {"vgpu_gb_direct": 20 * n}.get(kernel, 0)
    if name == "cp":  # the count pass reads the predicate columns, the write pass all three + the output
        return {"vgpu_mat_count": 16 * n, "vgpu_mat_write": 20 * n + 20 * passing}.get(kernel, 0)
    if name in ("c2", "c2dup"):
        build = wl.params["build_n"]
        return {"vgpu_gb_direct": 16 * n, "join_dense_table": 12 * build}.get(kernel, 0)
    if name == "c2b":
        return 8 * passing
    return 0


def query_bytes(name: str, wl, passing: int) -> float:
    """Algorithmic bytes of one whole query (inputs read once + outputs written once)."""
    if name == "cp":
        return 20.0 * wl.rows + 20.0 * passing
    if name == "c2b":
        return 8.0 * passing
    return wl.rows * wl.bytes_per_row


# ---- timing ------------------------------------------------------------------------------------------

def timed_blocks(step, steps: int, blocks: int, stream, world: int, sampler=None):
    """`blocks` timed blocks of exactly `steps` steps after half a second of busy lead-in, each
    bracketed by a barrier and a device synchronize, two untimed steps between blocks and no host-side
    work (the profiler's records are collected after the last block). Returns (per-block ms, launches
    per block, profile records, result of the last timed step -- the caller frees it)."""
    import torch
    from vectisdb_b200.engine import launch_count, profile_drain, profile_enable
    # the launch profiler's CUDA events are created here, untimed: in the timed blocks its records only
    # reuse them
    profile_enable(True)
    for _ in range(steps * blocks):
        step().free()
    torch.cuda.synchronize()
    profile_drain()
    profile_enable(False)
    t_hot = time.time()
    while time.time() - t_hot < 0.5:
        step().free()
    out, launches, last = [], 0, None
    if sampler:
        sampler.mark_begin()
    for b in range(blocks):
        for _ in range(2):
            step().free()
        if last is not None:
            last.free()
            last = None
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        profile_enable(True)
        l0 = launch_count()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(steps):
            r = step()
            if last is not None:
                last.free()
            last = r
        t1.record(stream)
        torch.cuda.synchronize()
        profile_enable(False)
        if world > 1:
            torch.distributed.barrier()
        ms = t0.elapsed_time(t1)
        out.append(max_over_ranks(ms, world) if world > 1 else ms)
        launches += launch_count() - l0
    if sampler:
        sampler.mark_end()
    return out, launches // blocks, profile_drain(), last


def kernel_table(prof):
    per = {}
    for kname, ms, nbytes, _rows in prof:
        d = per.setdefault(kname, [0.0, 0, 0])
        d[0] += ms
        d[1] += 1
        d[2] += nbytes
    return per


def roofline_of(name, wl, per, passing, groups):
    """The dominant kernel of the timed region against the measured HBM copy bandwidth."""
    total_ms = sum(v[0] for v in per.values()) or 1.0
    dom = max(per.items(), key=lambda kv: kv[1][0]) if per else ("none", [0.0, 1, 0])
    dom_avg_ms = dom[1][0] / max(1, dom[1][1])
    if dom[0] in ENGINE_COUNTED and dom[1][2] > 0:
        dom_bytes = dom[1][2] / max(1, dom[1][1])  # the engine's count for the launch (records written/read)
    else:
        dom_bytes = algorithmic_bytes(name, wl, dom[0], passing, groups)
    peak, peak_kind = hbm_peak()
    achieved = dom_bytes / (dom_avg_ms / 1000.0) / 1e9 if dom_avg_ms > 0 else 0.0
    traffic = None
    traffic_file = ROOT / "profiles" / f"traffic_{name}.json"
    if traffic_file.exists():
        traffic = json.loads(traffic_file.read_text()).get(dom[0])
    kernels = {k: {"launches": v[1], "ms": round(v[0], 4), "share": round(v[0] / total_ms, 4),
                   "avg_ms": round(v[0] / max(1, v[1]), 5)}
               for k, v in sorted(per.items(), key=lambda kv: -kv[1][0])}
    return {"bound": "hbm", "kernel": dom[0], "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
            "algorithmic_bytes": dom_bytes, "kernel_share": dom[1][0] / total_ms, "kernel_avg_ms": dom_avg_ms}, kernels


def cpu_baseline_of(name, wl, reps: int):
    """The oracle's OpenMP restatement timed on this host's cores over the whole table (warm, mean of
    `reps`); returns (baseline dict, the oracle's answer for the parity check)."""
    from oracle import oracle as O
    exp = oracle_result(name, wl)  # warm-up run, and the expected result
    t0 = time.perf_counter()
    for _ in range(reps):
        oracle_result(name, wl)
    dt = (time.perf_counter() - t0) / reps
    what = {"c2": "probe rows, build included", "c2dup": "probe rows, build included",
            "c2b": "pairs evaluated"}.get(name, "input rows")
    return ({"value": wl.rows / dt, "unit": "rows/s", "cores": O.threads(), "kind": "port",
             "label": CPU_BASELINE_LABEL, "ms_per_query": dt * 1000.0,
             "sample": f"the whole {name} table, the same one the GPU runs ({what}); mean of {reps} after a warm-up"},
            exp)


def measure_plain(name: str, args, world: int, rank: int, local: int, steps: int, blocks: int, e2e_steps: int,
                  cpu_reps: int, sample_clocks: bool):
    """One benchmark query with resident columns: timed blocks, roofline, e2e through the public API,
    the last timed result checked against the oracle, the CPU baseline. Returns the result dict."""
    import torch
    from vectisdb_b200 import ColumnCache, ExecuteOptions, GpuEngine, GpuTableRef, device_to_host

    wl = make_workload(name, pinned=True, rows=args.rows)
    engine = GpuEngine.instance()
    stream = torch.cuda.current_stream()
    # Every timed step does the whole query: derived structures the engine can keep across queries
    # (a join's dense table over a cached right side) are rebuilt each step; the kept-table figure is
    # measured separately below.
    os.environ["VGPU_JOIN_CACHE"] = "0"
    names_in_order = [c.name for c in wl.inputs]
    refs = []
    for table, cols in wl.tables.items():
        ref = GpuTableRef("memory", "main", table)
        ColumnCache.put_table(ref, [wl.inputs[names_in_order.index(c)] for c in cols])
        refs.append(ref)
    opts = ExecuteOptions(serve_whole_scan_from_cache=True, output_on_device=True, no_sync=True,
                          stream=stream.cuda_stream)

    def step():
        r = engine.execute_plan(wl.plan, [], opts)
        if not hasattr(r, "free"):
            raise RuntimeError(f"engine failed on {name}: {r.error_message}")
        return r

    sampler = ClockSampler(local) if sample_clocks else None
    if sampler:  # started before the warm-up, so its start-up lands in untimed work
        sampler.start()
    t_start = time.time()
    for _ in range(args.warmup):
        step().free()
    while time.time() - t_start < (1.0 if sampler else 0.2):
        step().free()
    blocks_ms, launches, prof, last = timed_blocks(step, steps, blocks, stream, world, sampler)
    clocks = sampler.stop() if sampler else None
    elapsed_ms = float(np.median(blocks_ms))
    value = wl.rows * steps * world / (elapsed_ms / 1000.0)
    # the last timed step's result, to the host for the parity check (outside the timed region)
    host = [device_to_host(c, stream.cuda_stream) for c in last.columns]
    last.free()
    groups = len(host[0]) if host else 0
    passing = wl.rows
    if name in ("c0", "c1"):
        passing = int(host[4 if name == "c1" else 2].sum())
    elif name in ("cp", "c2b"):
        passing = len(host[0])

    kept = None
    if name in ("c2", "c2dup"):
        # A repeated join keeps its dense right-side table (the engine's join-table cache): the same query
        # timed again with that reuse, reported beside the headline, never as it.
        os.environ["VGPU_JOIN_CACHE"] = "1"
        for _ in range(3):
            step().free()
        torch.cuda.synchronize()
        k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        k0.record(stream)
        lastk = None
        for _ in range(steps):
            r = step()
            if lastk is not None:
                lastk.free()
            lastk = r
        k1.record(stream)
        torch.cuda.synchronize()
        lastk.free()
        os.environ["VGPU_JOIN_CACHE"] = "0"
        kms = k0.elapsed_time(k1) / steps
        kept = {"ms_per_step": kms, "value": wl.rows * world / (kms / 1000.0),
                "note": "right-side dense table kept across steps (not the headline)"}
    for ref in refs:
        ColumnCache.invalidate_table(ref)

    per = kernel_table(prof)
    roofline, kernels = roofline_of(name, wl, per, passing, groups)
    peak = roofline["peak"]
    roofline["step_frac"] = query_bytes(name, wl, passing) / (elapsed_ms / steps / 1000.0) / 1e9 / peak

    # end to end through the public API: pinned host inputs, host result
    e2e_ms, d2h = [], 0
    h2d = sum(c.data.nbytes for c in wl.inputs)
    for i in range(e2e_steps + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = engine.execute_plan(wl.plan, wl.inputs)
        dt = time.perf_counter() - t0
        if not r.success:
            raise RuntimeError(r.error_message)
        if i > 0:
            e2e_ms.append(dt * 1000)
        d2h = sum(c.data.nbytes + (0 if c.validity is None else (len(c.validity) + 7) // 8) for c in r.columns)
        del r  # a caller that is done with a result lets it go before the next call
    e2e_value = wl.rows * world / (float(np.mean(e2e_ms)) / 1000.0) if e2e_ms else None

    cpu, parity = None, None
    if rank == 0 and cpu_reps > 0:
        cpu, exp = cpu_baseline_of(name, wl, cpu_reps)
        parity = parity_check(name, host, exp)
    elif rank == 0 and args.parity:
        parity = parity_check(name, host, oracle_result(name, wl))
    unit = "pairs/s" if name == "c2b" else "rows/s"
    if cpu:
        cpu["unit"] = unit
    out = {"metric": f"{name}_rows_per_s", "value": value, "unit": unit, "ms_per_step": elapsed_ms / steps,
           "steps": steps, "blocks_ms_per_step": [round(b / steps, 4) for b in blocks_ms],
           "config": {"workload": name, "rows": wl.rows, "bytes_per_row": wl.bytes_per_row,
                      "inputs": "resident in the device column cache (larger than L2, no flush needed)"
                      if name != "c2b" else "resident in the device column cache (32 KiB, L2-resident)",
                      "timing": f"median of {blocks} timed blocks of {steps} steps"},
           "parity": parity, "result_rows": groups, "passing_rows": passing,
           "roofline": roofline, "kernels": kernels,
           "e2e": {"value": e2e_value, "unit": unit, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                   "ms_per_step": float(np.mean(e2e_ms)) if e2e_ms else None},
           "gpu_launches": launches, "clocks": clocks, "cpu_baseline": cpu, "kept_join_table": kept}
    if name == "c2b":
        out["roofline"]["note"] = ("compute- and launch-bound: 32 KiB of inputs, 2^24 pairs evaluated; the HBM "
                                   "roofline only covers the matching pairs written")
    del wl
    gc.collect()
    return out


def measure_c3(args, world: int, rank: int, local: int, steps: int, blocks: int, cpu_queries: int,
               sample_clocks: bool):
    """Batching: 256 C0-shaped queries (own tables, constants and cardinalities) as one batched,
    graph-replayed call per step, against the plain loop of one vgpu_execute_plan per query. Every query
    of the last timed batched step is checked against the oracle and against its plain run."""
    import torch
    from oracle import oracle as O
    from vectisdb_b200 import BatchOptions, ColumnCache, ExecuteOptions, GpuEngine, GpuTableRef, device_to_host
    from vectisdb_b200 import workloads as W
    from vectisdb_b200.engine import launch_count, profile_drain, profile_enable

    wls = W.c3(n_queries=W.C3_QUERIES, pinned=True)
    engine = GpuEngine.instance()
    stream = torch.cuda.current_stream()
    refs = []
    for w in wls:
        for table in w.tables:
            ref = GpuTableRef("memory", "main", table)
            ColumnCache.put_table(ref, w.inputs)
            refs.append(ref)
    plans = [w.plan for w in wls]
    empty = [[] for _ in wls]
    rows = sum(w.rows for w in wls)
    opts = ExecuteOptions(serve_whole_scan_from_cache=True, output_on_device=True, stream=stream.cuda_stream)
    popts = ExecuteOptions(serve_whole_scan_from_cache=True, output_on_device=True, no_sync=True,
                           stream=stream.cuda_stream)
    prepared = engine.prepare_batch(plans)

    def batched_step():
        return engine.execute_batch(prepared, empty, opts)[0]

    def plain_step():
        out = []
        for pl in plans:
            r = engine.execute_plan(pl, [], popts)
            if not hasattr(r, "free"):
                raise RuntimeError(r.error_message)
            out.append(r)
        return out

    def free_all(rs):
        for r in rs:
            r.free()

    # warm-up: the autotuner measures its candidate geometries on this batch, then replays
    res, tuned = engine.execute_batch(prepared, empty, opts, BatchOptions(autotune=True))
    free_all(res)
    for _ in range(args.warmup):
        free_all(batched_step())
        free_all(plain_step())
    torch.cuda.synchronize()

    def timed(step_fn, nsteps, sampler):
        if sampler:
            sampler.start()
            t_s = time.time()
            while time.time() - t_s < 1.0:  # untimed until the sampler has settled
                free_all(step_fn())
        profile_enable(True)  # untimed: creates the profiler's events, which the timed steps reuse
        for _ in range(nsteps * blocks):
            free_all(step_fn())
        torch.cuda.synchronize()
        profile_drain()
        profile_enable(False)
        t_hot = time.time()
        while time.time() - t_hot < 0.5:
            free_all(step_fn())
        out, launches, last = [], 0, []
        if sampler:
            sampler.mark_begin()
        for _b in range(blocks):
            for _ in range(2):
                free_all(step_fn())
            free_all(last)
            last = []
            torch.cuda.synchronize()
            profile_enable(True)
            l0 = launch_count()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(nsteps):
                r = step_fn()
                free_all(last)
                last = r
            e1.record(stream)
            torch.cuda.synchronize()
            profile_enable(False)
            out.append(e0.elapsed_time(e1) / nsteps)
            launches += launch_count() - l0
        if sampler:
            sampler.mark_end()
        prof = profile_drain()
        return float(np.median(out)), launches // blocks, prof, (sampler.stop() if sampler else None), last

    b_ms, b_launches, b_prof, clocks, b_last = timed(batched_step, steps, ClockSampler(local) if sample_clocks else None)
    p_steps = max(3, steps // 5)
    p_ms, _, _, _, p_last = timed(plain_step, p_steps, None)

    # identical results: every query of the last batched step against its plain run and the oracle
    match_plain, match_oracle = True, True
    for w, a, b in zip(wls, b_last, p_last):
        ha = [device_to_host(c, stream.cuda_stream) for c in a.columns]
        hb = [device_to_host(c, stream.cuda_stream) for c in b.columns]
        oa, ob = np.argsort(ha[0]), np.argsort(hb[0])
        for i, (x, y) in enumerate(zip(ha, hb)):
            match_plain &= _close(x[oa], y[ob]) if i == 1 else bool(np.array_equal(x[oa], y[ob]))
        match_oracle &= parity_check("c0", ha, O.c0(*[c.data for c in w.inputs], w.params["v_lt"], w.params["w_mod"]))
    free_all(b_last)
    free_all(p_last)

    per = kernel_table(b_prof)
    total_ms = sum(v[0] for v in per.values()) or 1.0
    dom = max(per.items(), key=lambda kv: kv[1][0])
    dom_avg_ms = dom[1][0] / max(1, dom[1][1])
    peak, peak_kind = hbm_peak()
    achieved = 20 * rows / (dom_avg_ms / 1000.0) / 1e9

    # end to end: host (pinned) inputs through the public batch call, host results
    e2e_ms, d2h = [], 0
    host_inputs = [w.inputs for w in wls]
    for i in range(args.e2e_steps + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res, _ = engine.execute_batch(plans, host_inputs, ExecuteOptions(stream=stream.cuda_stream))
        dt = time.perf_counter() - t0
        if i > 0:
            e2e_ms.append(dt * 1000)
        d2h = sum(c.data.nbytes for r in res for c in r.columns)
    h2d = sum(c.data.nbytes for w in wls for c in w.inputs)

    cpu = None
    if rank == 0 and cpu_queries > 0:
        sample = wls[: min(len(wls), cpu_queries)]
        t0 = time.perf_counter()
        for w in sample:
            O.c0(w.inputs[0].data, w.inputs[1].data, w.inputs[2].data, w.params["v_lt"], w.params["w_mod"])
        dt = time.perf_counter() - t0
        cpu = {"value": sum(w.rows for w in sample) / dt, "unit": "rows/s", "cores": O.threads(), "kind": "port",
               "label": CPU_BASELINE_LABEL,
               "sample": f"the first {len(sample)} of the {len(wls)} queries, run one after another"}
    for ref in refs:
        ColumnCache.invalidate_table(ref)
    out = {
        "metric": "c3_rows_per_s", "value": rows / (b_ms / 1000.0), "unit": "rows/s", "ms_per_step": b_ms,
        "steps": steps,
        "config": {"workload": "c3", "queries": len(wls), "rows": rows, "bytes_per_row": 20.0,
                   "inputs": "resident in the device column cache (larger than L2, no flush needed)",
                   "geometry": {k: tuned[k] for k in ("block", "items", "tile_rows", "smem_slots")},
                   "timing": f"median of {blocks} timed blocks of {steps} steps"},
        "plain": {"value": rows / (p_ms / 1000.0), "ms_per_step": p_ms, "steps": p_steps,
                  "form": "one vgpu_execute_plan per query, device outputs, no per-query sync"},
        "batched_over_plain": p_ms / b_ms,
        "results_match_plain": bool(match_plain),
        "parity": bool(match_oracle),
        "roofline": {"bound": "hbm", "kernel": dom[0], "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                     "algorithmic_bytes": 20 * rows, "kernel_share": dom[1][0] / total_ms, "kernel_avg_ms": dom_avg_ms},
        "kernels": {k: {"launches": v[1], "ms": round(v[0], 4), "share": round(v[0] / total_ms, 4)}
                    for k, v in sorted(per.items(), key=lambda kv: -kv[1][0])},
        "e2e": {"value": rows / (float(np.mean(e2e_ms)) / 1000.0) if e2e_ms else None, "unit": "rows/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": float(np.mean(e2e_ms)) if e2e_ms else None},
        "gpu_launches": b_launches,
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    del wls
    gc.collect()
    return out


def measure_c4(args, world: int, rank: int, local: int, rates, n_req: int, sample_clocks: bool):
    """Serving: an open-loop Poisson trace of a seeded mix (50% c0-, 30% c1-, 20% c2-shaped queries,
    each over the first 2^12..2^26 rows of a resident base table) at a sweep of arrival rates, served
    by the engine's server (slots, memory-budget admission, same-template batching) and by the serial
    executor (one request at a time). Latency = submit -> completion; throughput = rows / makespan.
    Every request's result in the served run is checked against its result in the serial run."""
    import threading
    import torch
    from vectisdb_b200 import ColumnCache, ExecuteOptions, GpuTableRef, Server, device_to_host
    from vectisdb_b200 import workloads as W
    from vectisdb_b200.engine import launch_count

    base_log2 = 26 if not args.rows else int(np.log2(args.rows))
    c0 = W.c0(n=1 << base_log2, seed=40, table="c4_c0")
    c1 = W.c1(n=1 << base_log2, seed=41, table="c4_c1")
    c2 = W.c2(probe_n=1 << base_log2, build_n=1 << 24, seed=42)
    refs = []
    for wl in (c0, c1, c2):
        names = [c.name for c in wl.inputs]
        for table, cols in wl.tables.items():
            ref = GpuTableRef("memory", "main", table)
            ColumnCache.put_table(ref, [wl.inputs[names.index(c)] for c in cols])
            refs.append(ref)
    dcol = ColumnCache.device_column
    t_c0, t_c1 = GpuTableRef("memory", "main", "c4_c0"), GpuTableRef("memory", "main", "c4_c1")
    t_p, t_b = GpuTableRef("memory", "main", "c2_probe"), GpuTableRef("memory", "main", "c2_build")

    rng = np.random.default_rng(4)
    trace = []  # (kind, plan, inputs, rows)
    for i in range(n_req):
        kind = rng.choice(["c0", "c1", "c2"], p=[0.5, 0.3, 0.2])
        rows = int(round(2 ** rng.uniform(12, base_log2)))
        if kind == "c0":
            plan = W.c0_plan(float(np.round(rng.uniform(0.1, 0.9), 6)), int(rng.integers(2, 17)))
            ins = [dcol(t_c0, n, rows) for n in ("k", "v", "w")]
        elif kind == "c1":
            plan = W.c1_plan(c1.params["ts_gt"])
            ins = [dcol(t_c1, n, rows) for n in ("a", "b", "amt", "v", "ts")]
        else:
            plan = W.c2_plan()
            ins = [dcol(t_p, "pkey", rows), dcol(t_p, "x", rows), dcol(t_b, "bkey"), dcol(t_b, "g")]
        trace.append((kind, plan, ins, rows))
    total_rows = sum(t[3] for t in trace)
    gaps = rng.exponential(1.0, n_req)  # unit-rate Poisson arrivals, scaled per rate

    def serve(rate, slots, batch_max, keep=False, on_device=False):
        srv = Server(slots=slots, batch_max=batch_max)
        sub_opts = ExecuteOptions(output_on_device=on_device)
        arrivals = np.cumsum(gaps) / rate
        done = [None] * n_req
        results = [None] * n_req
        t0 = time.perf_counter()
        submit_t = [0.0] * n_req
        ids = [0] * n_req

        def collector():
            for i in range(n_req):
                while ids[i] == 0:
                    time.sleep(0.0002)
                res, info = srv.wait(ids[i])
                done[i] = info
                if res is not None:
                    if keep:
                        results[i] = [device_to_host(c) if c.data is None else np.array(c.data, copy=True)
                                      for c in res.columns]
                    if hasattr(res, "free"):
                        res.free()

        th = threading.Thread(target=collector)
        th.start()
        for i, (kind, plan, ins, rows) in enumerate(trace):
            delay = arrivals[i] - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            submit_t[i] = time.perf_counter() - t0
            ids[i] = srv.submit(plan, ins, sub_opts)
        th.join()
        st = srv.stats()
        srv.close()
        lat = np.array([d["queued_ms"] + d["run_ms"] for d in done])
        finish = max(submit_t[i] + lat[i] / 1000.0 for i in range(n_req))
        failed = sum(1 for d in done if d["status"] != 0)
        return {"rate_per_s": rate, "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "rows_per_s": total_rows / finish, "makespan_s": finish, "failed": failed,
                "batches": st["batches"], "batched_requests": st["batched_requests"],
                "peak_in_flight": st["peak_in_flight"], "peak_reserved_gb": st["peak_reserved_bytes"] / 1e9}, results

    def same(a, b):
        """One request's result in the mix against its serial run (columns in engine order)."""
        if a is None or b is None or len(a) != len(b):
            return False
        o_a, o_b = np.lexsort(a[:2][::-1]) if len(a) > 5 else np.argsort(a[0]), \
            np.lexsort(b[:2][::-1]) if len(b) > 5 else np.argsort(b[0])
        for x, y in zip(a, b):
            x, y = x[o_a], y[o_b]
            if x.dtype.kind == "f":
                if not _close(x, y):
                    return False
            elif not np.array_equal(x, y):
                return False
        return True

    # warm-up: every kernel shape of the mix compiled, the memory pool grown to the mix's peak; the
    # served and the serial results of every request are compared here
    served_info, served_res = serve(1e6, 8, 64, keep=True)
    serial_info, serial_res = serve(1e6, 1, 1, keep=True)
    mismatched = [i for i, (a, b) in enumerate(zip(served_res, serial_res)) if not same(a, b)]
    results_match = not mismatched
    mismatch_examples = [{"request": i, "kind": trace[i][0], "rows": trace[i][3],
                          "served_rows": None if served_res[i] is None else len(served_res[i][0]),
                          "serial_rows": None if serial_res[i] is None else len(serial_res[i][0])}
                         for i in mismatched[:4]]
    failed_warmup = {"served": served_info["failed"], "serial": serial_info["failed"]}
    del served_res, serial_res
    sampler = ClockSampler(local) if sample_clocks else None
    if sampler:
        sampler.start()
        sampler.mark_begin()
    l0 = launch_count()
    sweep = []
    for r in rates:
        served, _ = serve(r, 8, 64)
        serial, _ = serve(r, 1, 1)
        sweep.append({"rate_per_s": r, "served": served, "serial": serial})
    # the same saturating trace with results left in device memory (no device->host copy of the 1.5 GB
    # of group results): what the GPU work alone allows
    top_rate = rates[-1]
    dev = {"served": serve(top_rate, 8, 64, on_device=True)[0], "serial": serve(top_rate, 1, 1, on_device=True)[0]}
    launches = launch_count() - l0
    clocks = None
    if sampler:
        sampler.mark_end()
        clocks = sampler.stop()
    for ref in refs:
        ColumnCache.invalidate_table(ref)
    top = sweep[-1]
    out = {
        "metric": "c4_rows_per_s", "value": top["served"]["rows_per_s"], "unit": "rows/s",
        "ms_per_step": top["served"]["makespan_s"] * 1000.0, "steps": len(rates),
        "config": {"workload": "c4", "requests": n_req, "rows": total_rows, "mix": "50% c0, 30% c1, 20% c2 shaped",
                   "rows_per_request": f"log-uniform 2^12..2^{base_log2} prefixes of resident base tables",
                   "admission_budget_gb": 120, "slots": 8, "batch_max": 64,
                   "inputs": "resident in the device column cache",
                   "results": "host memory (page-locked, handed to the client without a copy)"},
        "p50_ms": top["served"]["p50_ms"], "p99_ms": top["served"]["p99_ms"],
        "serial": {"rows_per_s": top["serial"]["rows_per_s"], "p50_ms": top["serial"]["p50_ms"],
                   "p99_ms": top["serial"]["p99_ms"]},
        "served_over_serial": top["served"]["rows_per_s"] / top["serial"]["rows_per_s"],
        "device_outputs": {"rate_per_s": top_rate, "served": dev["served"], "serial": dev["serial"],
                           "served_over_serial": dev["served"]["rows_per_s"] / dev["serial"]["rows_per_s"]},
        "results_match_serial": bool(results_match),
        "mismatches": len(mismatched), "mismatch_examples": mismatch_examples, "failed_in_comparison": failed_warmup,
        "sweep": sweep,
        "e2e": None,
        "gpu_launches": launches,
        "clocks": clocks,
        "cpu_baseline": None,
    }
    del c0, c1, c2, trace
    gc.collect()
    return out


class _Share:
    """A sharded step's output columns (torch tensors), dropped by free() like an engine result."""

    def __init__(self, cols):
        self.cols = cols

    def free(self):
        self.cols = None


def measure_sharded(args, world: int, rank: int, local: int, steps: int, blocks: int, sample_clocks: bool):
    """c1 as ONE query split by rows across the ranks: rank r holds its own slice of 2^27 rows (rank 0's
    is the one-GPU c1 table, seed 1; rank r > 0 draws from seed 1 + r), runs the GROUP BY on it, and the
    partial groups are merged on the GPUs (distributed.device_sharded_group_by: routing kernel, NCCL
    all-to-all of device rows, engine re-aggregation, finish kernels). Every timed step is the whole
    distributed query; value = rows of all ranks / time (max over ranks). Parity: at one rank, the
    merged groups against the oracle on the same table."""
    import datetime
    import socket
    import torch.distributed as dist
    own_group = not dist.is_initialized()
    if own_group:  # one GPU: a one-rank nccl group, so the exchange runs as it does on N ranks
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                                timeout=datetime.timedelta(seconds=120))
    try:
        return _measure_sharded(args, world, rank, local, steps, blocks, sample_clocks)
    finally:
        if own_group:
            dist.destroy_process_group()


def _measure_sharded(args, world, rank, local, steps, blocks, sample_clocks):
    import torch
    from vectisdb_b200 import ColumnCache, GpuTableRef
    from vectisdb_b200 import workloads as W
    from vectisdb_b200.distributed import device_sharded_group_by
    from vectisdb_b200.engine import GpuValueType as T

    rows = args.rows or W.C1_ROWS
    wl = W.c1(n=rows, seed=1 + rank, pinned=True, table="c1_shard")
    ref = GpuTableRef("memory", "main", "c1_shard")
    ColumnCache.put_table(ref, wl.inputs)
    cols = [ColumnCache.device_column(ref, c.name, rows) for c in wl.inputs]
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        def step():
            return _Share(device_sharded_group_by(wl.plan, cols, {"v": T.FLOAT64}))

        sampler = ClockSampler(local) if sample_clocks else None
        if sampler:
            sampler.start()
        t_start = time.time()
        for _ in range(args.warmup):
            step().free()
        while time.time() - t_start < (1.0 if sampler else 0.2):
            step().free()
        blocks_ms, launches, prof, last = timed_blocks(step, steps, blocks, side, world, sampler)
        clocks = sampler.stop() if sampler else None
        host = [(name, t.cpu().numpy()) for name, t in last.cols]
        last.free()
    elapsed_ms = float(np.median(blocks_ms))
    value = rows * steps * world / (elapsed_ms / 1000.0)
    groups = len(host[0][1]) if host else 0
    passing = int(host[4][1].sum()) if host else 0
    parity = None
    if world == 1 and args.parity:
        d = dict(host)
        order = np.lexsort((d["b"], d["a"]))
        s = d["agg_0"][order]
        hug = np.empty(len(order), dtype=[("lower", "<u8"), ("upper", "<i8")])
        hug["lower"], hug["upper"] = s[:, 0].view(np.uint64), s[:, 1]
        parity = parity_check("c1", [d["a"][order], d["b"][order], hug, d["agg_1"][order], d["agg_2"][order],
                                     d["agg_3"][order]], oracle_result("c1", wl))
    ColumnCache.invalidate_table(ref)
    per = kernel_table(prof)
    roofline, kernels = roofline_of("c1", wl, per, passing, groups)
    exchange = {k: v for k, v in kernels.items() if k.startswith("shard_")}
    out = {"metric": "c1_rows_per_s", "value": value, "unit": "rows/s", "ms_per_step": elapsed_ms / steps,
           "steps": steps, "blocks_ms_per_step": [round(b / steps, 4) for b in blocks_ms],
           "config": {"workload": "c1", "rows": rows * world, "rows_per_rank": rows, "bytes_per_row": 32.0,
                      "inputs": "resident in the device column cache (larger than L2, no flush needed)",
                      "timing": f"median of {blocks} timed blocks of {steps} steps",
                      "merge": "partial groups routed to owner ranks, NCCL all-to-all of device rows, "
                               "engine re-aggregation"},
           "parity": parity, "result_rows_rank0": groups, "roofline": roofline, "kernels": kernels,
           "exchange_kernels": exchange, "e2e": None, "gpu_launches": launches, "clocks": clocks,
           "cpu_baseline": None}
    del wl
    gc.collect()
    return out


def run_reference(args, world, rank):
    """The reference arm: the CPU restatement of the query (oracle/oracle.cpp, OpenMP, every host
    core) on the same full-size table the GPU arm runs, timed per step like it. Rank 0 only."""
    if rank != 0:
        return
    from oracle import oracle as O
    name = args.config
    cores = O.threads()
    if name == "c3":
        from vectisdb_b200 import workloads as W
        wls = W.c3()
        sample = sum(w.rows for w in wls)
        fn = lambda: [O.c0(w.inputs[0].data, w.inputs[1].data, w.inputs[2].data, w.params["v_lt"],  # noqa: E731
                           w.params["w_mod"]) for w in wls]
        desc = "the 256 c3 queries, one after another (the whole batch)"
        unit = "rows/s"
    elif name == "c4":
        print(json.dumps({"impl": "reference", "metric": "c4_rows_per_s",
                          "unavailable": "serving has no CPU reference form: the serial GPU executor is its baseline"}))
        return
    else:
        wl = make_workload(name, pinned=False, rows=args.rows)
        sample = wl.rows
        fn = lambda: oracle_result(name, wl)  # noqa: E731
        desc = f"the whole {name} table, the same one the GPU arm runs"
        unit = "pairs/s" if name == "c2b" else "rows/s"
    for _ in range(args.warmup):
        fn()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        fn()
    dt = time.perf_counter() - t0
    value = sample * args.steps / dt
    line = {"metric": f"{name}_rows_per_s", "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt * 1000 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64/f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": name, "rows": sample, "rows_per_step": sample, "parallelism": "host threads"},
            "cpu_baseline": {"value": value, "unit": unit, "cores": cores, "kind": "port", "label": CPU_BASELINE_LABEL,
                             "sample": desc},
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--config", default="c1", choices=list(PLAIN_CONFIGS) + ["c3", "c4"])
    p.add_argument("--e2e-steps", type=int, default=5)
    p.add_argument("--blocks", type=int, default=7, help="timed blocks of --steps steps; the median is reported")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-parity", dest="parity", action="store_false",
                   help="skip the oracle check of the last timed step (small profiling runs)")
    p.add_argument("--per-config", choices=["auto", "on", "off"], default="auto",
                   help="also measure every other query (auto: with the c1 headline at full size on one GPU)")
    p.add_argument("--rows", type=int, default=0, help="small-case size for profiling (0 = the full workload)")
    p.add_argument("--mode", choices=["replicas", "sharded"], default="replicas",
                   help="N>1: independent replicas of the query (default), or c1 as one query split by rows "
                        "across the ranks with the partial groups merged on the GPUs")
    args = p.parse_args()
    world, rank, local = dist_setup()

    if args.impl == "reference":
        run_reference(args, world, rank)
        return

    import torch
    torch.cuda.set_device(local)
    # One dedicated stream for the engine and the timing events alike: torch's default stream has the
    # handle 0, which the engine takes as "its own stream", and events on another stream than the
    # kernels' would time only the host's enqueueing of calls that return without a sync.
    torch.cuda.set_stream(torch.cuda.Stream())
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from vectisdb_b200 import ColumnCache
    from vectisdb_b200.abi import lib
    lib().vgpu_set_device(local)
    ColumnCache.init(0.6)

    name = args.config
    cpu_reps = 0 if args.no_cpu_baseline or rank != 0 else (2 if name in ("c1", "c2", "c2dup") else 3)
    if args.mode == "sharded":
        if name != "c1":
            raise SystemExit("--mode sharded runs the c1 query")
        line = measure_sharded(args, world, rank, local, args.steps, args.blocks, True)
    elif name == "c3":
        line = measure_c3(args, world, rank, local, args.steps, args.blocks, 0 if args.no_cpu_baseline else 64, True)
    elif name == "c4":
        rates = [50.0, 100.0, 200.0, 400.0, 800.0, 1600.0, 3200.0, 6400.0, 12800.0, 25600.0]
        line = measure_c4(args, world, rank, local, rates, 160 if not args.rows else 40, True)
    else:
        line = measure_plain(name, args, world, rank, local, args.steps, args.blocks, args.e2e_steps, cpu_reps, True)
    line.update({"n_gpus": world, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                 "vs_baseline": None, "dtype": "int64/f64", "data": "synthetic"})
    line["config"]["parallelism"] = f"row-sharded x{world}" if args.mode == "sharded" else f"replicas x{world}"
    per_config = args.per_config == "on" or (args.per_config == "auto" and name == "c1" and world == 1 and not args.rows
                                             and args.mode == "replicas")
    if per_config:
        per = {}
        for other in PER_CONFIG_ORDER:
            if other == name:
                continue
            t0 = time.time()
            try:
                if other == "c1_sharded":
                    per[other] = measure_sharded(args, world, rank, local, 10, 3, False)
                elif other == "c3":
                    per[other] = measure_c3(args, world, rank, local, 10, 3, 64 if cpu_reps else 0, False)
                elif other == "c4":
                    per[other] = measure_c4(args, world, rank, local, [200.0, 1600.0, 25600.0], 160, False)
                else:
                    per[other] = measure_plain(other, args, world, rank, local, 10 if other == "c2dup" else 20, 3,
                                               2, 1 if cpu_reps else 0, False)
            except Exception as e:  # a failing secondary query is reported, not fatal to the headline
                per[other] = {"error": f"{type(e).__name__}: {e}"}
            per[other]["wall_s"] = round(time.time() - t0, 1)
        line["per_config"] = per
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
