"""Python entry points of the oracle (TEST INFRASTRUCTURE ONLY).

The oracle is the CPU restatement of the benchmark queries (oracle.cpp, OpenMP) plus the plan-level
evaluator (plan_oracle.py). Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
use it, always as the checker or the timed CPU baseline, never as the thing measured on the GPU.

Pinning: plan_oracle is checked against the known answers of the reference engine's own test suite
(cuda_engine/tests/test_gpu_executor.cpp), re-expressed as fixtures in tests/golden/; the config
functions here are checked against plan_oracle on the same seeded inputs (tests/test_oracle.py).
DuckDB itself is not installed in this image, so parity with DuckDB's CPU execution rests on this
restatement of its semantics.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
_L = None


def lib() -> C.CDLL:
    global _L
    if _L is None:
        if not LIB.exists():
            subprocess.run(["make", "-C", str(HERE)], check=True, capture_output=True)
        L = C.CDLL(str(LIB))
        vp, u64, i64 = C.c_void_p, C.c_uint64, C.c_int64
        L.oracle_c0.argtypes = [vp, vp, vp, u64, C.c_double, i64, vp, vp, vp, vp, vp, u64]
        L.oracle_c0.restype = i64
        L.oracle_c1.argtypes = [vp, vp, vp, vp, vp, u64, i64, vp, vp, vp, vp, vp, vp, vp, u64]
        L.oracle_c1.restype = i64
        L.oracle_c2.argtypes = [vp, vp, u64, vp, vp, u64, vp, vp, vp, u64]
        L.oracle_c2.restype = i64
        L.oracle_c2b.argtypes = [vp, u64, vp, u64, C.c_int32, vp, vp, u64]
        L.oracle_cp.argtypes = [vp, vp, vp, u64, C.c_double, i64, vp, vp, vp, u64]
        L.oracle_cp.restype = i64
        L.oracle_c2b.restype = i64
        L.oracle_threads.restype = C.c_int
        L.oracle_set_threads.argtypes = [C.c_int]
        _L = L
    return _L


def threads() -> int:
    return lib().oracle_threads()


def set_threads(n: int) -> None:
    lib().oracle_set_threads(n)


def _p(a: np.ndarray):
    return a.ctypes.data


def c0(k, v, w, v_lt=0.5, w_mod=7, capacity=None):
    """-> dict(k, sum, count, min, max), sorted by k."""
    cap = capacity or 1 << 20
    out = {"k": np.empty(cap, "<i4"), "sum": np.empty(cap, "<f8"), "count": np.empty(cap, "<i8"),
           "min": np.empty(cap, "<i8"), "max": np.empty(cap, "<i8")}
    g = lib().oracle_c0(_p(k), _p(v), _p(w), len(k), v_lt, w_mod, _p(out["k"]), _p(out["sum"]), _p(out["count"]),
                        _p(out["min"]), _p(out["max"]), cap)
    if g < 0:
        raise RuntimeError("oracle c0: capacity too small")
    return {key: val[:g] for key, val in out.items()}


def cp(k, v, w, v_lt=0.5, w_mod=7):
    """-> dict(k, v, w): the passing rows of the filter, projected (v*2+1), in input order."""
    L = lib()
    n = L.oracle_cp(_p(k), _p(v), _p(w), len(k), v_lt, w_mod, None, None, None, 0)
    out = {"k": np.empty(max(n, 1), "<i4"), "v": np.empty(max(n, 1), "<f8"), "w": np.empty(max(n, 1), "<i8")}
    L.oracle_cp(_p(k), _p(v), _p(w), len(k), v_lt, w_mod, _p(out["k"]), _p(out["v"]), _p(out["w"]), n)
    return {key: val[:n] for key, val in out.items()}


def c1(a, b, amt, v, ts, ts_gt, capacity=None):
    """-> dict(a, b, sum_lo, sum_hi, avg, count, max), sorted by (a, b)."""
    cap = capacity or len(a)
    out = {"a": np.empty(cap, "<i4"), "b": np.empty(cap, "<i4"), "sum_lo": np.empty(cap, "<u8"),
           "sum_hi": np.empty(cap, "<i8"), "avg": np.empty(cap, "<f8"), "count": np.empty(cap, "<i8"),
           "max": np.empty(cap, "<i8")}
    g = lib().oracle_c1(_p(a), _p(b), _p(amt), _p(v), _p(ts), len(a), ts_gt, _p(out["a"]), _p(out["b"]),
                        _p(out["sum_lo"]), _p(out["sum_hi"]), _p(out["avg"]), _p(out["count"]), _p(out["max"]), cap)
    if g < 0:
        raise RuntimeError("oracle c1: capacity too small")
    return {key: val[:g] for key, val in out.items()}


def c2(bkey, bg, pkey, px, capacity=1 << 20):
    """-> dict(g, sum, count), sorted by g."""
    out = {"g": np.empty(capacity, "<i4"), "sum": np.empty(capacity, "<f8"), "count": np.empty(capacity, "<i8")}
    g = lib().oracle_c2(_p(bkey), _p(bg), len(bkey), _p(pkey), _p(px), len(pkey), _p(out["g"]), _p(out["sum"]),
                        _p(out["count"]), capacity)
    if g < 0:
        raise RuntimeError("oracle c2: capacity too small")
    return {key: val[:g] for key, val in out.items()}


def c2b(a, b, modulus=13, count_only=False):
    """-> (count, a_out, b_out) in left-major order."""
    L = lib()
    total = L.oracle_c2b(_p(a), len(a), _p(b), len(b), modulus, None, None, 0)
    if count_only:
        return int(total), None, None
    oa = np.empty(max(total, 1), "<i4")
    ob = np.empty(max(total, 1), "<i4")
    L.oracle_c2b(_p(a), len(a), _p(b), len(b), modulus, _p(oa), _p(ob), total)
    return int(total), oa[:total], ob[:total]
