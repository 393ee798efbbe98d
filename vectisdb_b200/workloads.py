"""Seeded synthetic tables and the plans of the benchmark queries.

Every generator is a pure function of (seed, column id, row) (libvgpu_datagen.so), so any size of a
configuration is a prefix-stable, reproducible table. Plans are built the way the DuckDB extension's
translator lowers the SQL (extension/src/expression_translator.cpp:287-493): expressions are CUDA
statements reading ((const T*)inputs[i])[row] and writing ((T*)out)[idx]; projections name their
outputs col<i>; aggregates are named agg_<i>.

Configurations (sizes are the full benchmark sizes; tests use smaller `n`):
  c0  filter + group-by: k INT32 U[0,1024), v DOUBLE U[0,1), w BIGINT U[0,1e6), 2^24 rows, seed 0
      SELECT k, SUM(v*2+1), COUNT(*), MIN(w), MAX(w) WHERE v<0.5 AND w%7<>0 GROUP BY k
  c1  high-cardinality group-by: a INT32 Zipf(1.1) over 2^20, b INT32 U[0,16), amt DECIMAL(18,2)
      as BIGINT cents U[0,1e6), v DOUBLE U[0,1), ts BIGINT U[0,2^62), 2^27 rows, seed 1
      SELECT a, b, SUM(amt), AVG(v), COUNT(*), MAX(ts) WHERE ts > median(ts) GROUP BY a, b
  c2  join + aggregate: build key = permutation of [0,2^24), g INT32 U[0,4096); probe 2^28 rows,
      key 90% a build key at a Zipf(0.8) rank, 10% U[2^24, 2^25); x DOUBLE U[0,1), seed 2
      SELECT b.g, SUM(p.x) FROM probe p JOIN build b ON p.key = b.key GROUP BY b.g
  c2b filtered cross product: 4096 x 4096, a, b INT32 U[0,2^20), seed 5
      SELECT l.a, r.b FROM l, r WHERE (l.a + r.b) % 13 = 0
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from .engine import (GpuAggregateKind as A, GpuColumn, GpuPlanNode, GpuTableRef, GpuValueType as T,
                     make_aggregate, make_column, make_cross_product, make_expr, make_filter, make_group_by,
                     make_join, make_projection, make_scan)

_DG = None


def datagen() -> C.CDLL:
    global _DG
    if _DG is None:
        path = Path(__file__).resolve().parent / "libvgpu_datagen.so"
        if not path.exists():
            raise RuntimeError(f"{path} is missing: build it with `python -m vectisdb_b200.build`")
        lib = C.CDLL(str(path))
        u64, u32, i64, vp = C.c_uint64, C.c_uint32, C.c_int64, C.c_void_p
        lib.vgdg_uniform_i32.argtypes = [u64, u32, u64, u64, i64, i64, vp]
        lib.vgdg_uniform_i64.argtypes = [u64, u32, u64, u64, i64, u64, vp]
        lib.vgdg_uniform_f64.argtypes = [u64, u32, u64, u64, vp]
        lib.vgdg_zipf_cdf.argtypes = [u64, C.c_double, vp]
        lib.vgdg_zipf_i64.argtypes = [u64, u32, u64, u64, vp, u64, vp]
        lib.vgdg_zipf_i32.argtypes = [u64, u32, u64, u64, vp, u64, vp]
        lib.vgdg_permutation_i64.argtypes = [u64, u32, u64, vp]
        lib.vgdg_probe_keys_i64.argtypes = [u64, u32, u64, u64, vp, vp, u64, C.c_double, i64, u64, vp]
        lib.vgdg_median_i64.argtypes = [vp, u64]
        lib.vgdg_median_i64.restype = i64
        for f in (lib.vgdg_uniform_i32, lib.vgdg_uniform_i64, lib.vgdg_uniform_f64, lib.vgdg_zipf_cdf,
                  lib.vgdg_zipf_i64, lib.vgdg_zipf_i32, lib.vgdg_permutation_i64, lib.vgdg_probe_keys_i64):
            f.restype = None
        _DG = lib
    return _DG


def _alloc(n: int, dtype, pinned: bool):
    if pinned:
        import torch  # plumbing only: page-locked host buffers for the end-to-end copies
        t = torch.empty(n, dtype={np.dtype("<i4"): torch.int32, np.dtype("<i8"): torch.int64,
                                  np.dtype("<f8"): torch.float64}[np.dtype(dtype)], pin_memory=True)
        return t.numpy()
    return np.empty(n, dtype=dtype)


def uniform_i32(seed, col, n, lo, hi, offset=0, pinned=False):
    out = _alloc(n, "<i4", pinned)
    datagen().vgdg_uniform_i32(seed, col, offset, n, lo, hi, out.ctypes.data)
    return out


def uniform_i64(seed, col, n, lo, span, offset=0, pinned=False):
    out = _alloc(n, "<i8", pinned)
    datagen().vgdg_uniform_i64(seed, col, offset, n, lo, span, out.ctypes.data)
    return out


def uniform_f64(seed, col, n, offset=0, pinned=False):
    out = _alloc(n, "<f8", pinned)
    datagen().vgdg_uniform_f64(seed, col, offset, n, out.ctypes.data)
    return out


_CDF_CACHE: dict = {}


def zipf_cdf(values: int, s: float) -> np.ndarray:
    key = (values, s)
    if key not in _CDF_CACHE:
        cdf = np.empty(values, dtype="<f8")
        datagen().vgdg_zipf_cdf(values, s, cdf.ctypes.data)
        _CDF_CACHE[key] = cdf
    return _CDF_CACHE[key]


def zipf_i32(seed, col, n, values, s, offset=0, pinned=False):
    cdf = zipf_cdf(values, s)
    out = _alloc(n, "<i4", pinned)
    datagen().vgdg_zipf_i32(seed, col, offset, n, cdf.ctypes.data, values, out.ctypes.data)
    return out


def permutation_i64(seed, col, n, pinned=False):
    out = _alloc(n, "<i8", pinned)
    datagen().vgdg_permutation_i64(seed, col, n, out.ctypes.data)
    return out


def median_i64(values: np.ndarray) -> int:
    v = np.ascontiguousarray(values, dtype="<i8")
    return int(datagen().vgdg_median_i64(v.ctypes.data, len(v)))


# ---- configurations ------------------------------------------------------------------------------

@dataclass
class Workload:
    name: str
    plan: GpuPlanNode
    inputs: list[GpuColumn]           # scan inputs, traversal order
    rows: int                         # rows counted by the metric (input rows; probe rows for joins)
    bytes_per_row: float              # algorithmic input bytes per counted row
    params: dict = field(default_factory=dict)
    tables: dict = field(default_factory=dict)  # table ref -> scan input names (for the column cache)


C0_ROWS = 1 << 24
C1_ROWS = 1 << 27
C2_BUILD_ROWS = 1 << 24
C2_PROBE_ROWS = 1 << 28
C2B_SIDE = 4096


def c0_plan(v_lt: float = 0.5, w_mod: int = 7, table: GpuTableRef | None = None) -> GpuPlanNode:
    scan = make_scan(["k", "v", "w"], table or GpuTableRef("memory", "main", "c0"))
    filt = make_filter([
        make_expr(f"((bool*)out)[idx] = (((const double*)inputs[0])[row] < {float(v_lt)!r});", ["v"], T.BOOLEAN),
        make_expr(f"((bool*)out)[idx] = ((((const long long*)inputs[0])[row] % {int(w_mod)}LL) != 0LL);", ["w"],
                  T.BOOLEAN),
    ], scan)
    proj = make_projection([
        make_expr("((int*)out)[idx] = ((const int*)inputs[0])[row];", ["k"], T.INT32),
        make_expr("((double*)out)[idx] = ((((const double*)inputs[0])[row] * 2.0) + 1.0);", ["v"], T.FLOAT64),
        make_expr("((long long*)out)[idx] = ((const long long*)inputs[0])[row];", ["w"], T.INT64),
    ], filt)
    return make_group_by(["col0"], [
        make_aggregate(A.SUM, "col1", T.FLOAT64),
        make_aggregate(A.COUNT_STAR, "", T.INT64),
        make_aggregate(A.MIN, "col2", T.INT64),
        make_aggregate(A.MAX, "col2", T.INT64),
    ], proj)


def c0(n: int = C0_ROWS, seed: int = 0, k_card: int = 1024, v_lt: float = 0.5, w_mod: int = 7,
       pinned: bool = False, table: str = "c0") -> Workload:
    k = uniform_i32(seed, 0, n, 0, k_card, pinned=pinned)
    v = uniform_f64(seed, 1, n, pinned=pinned)
    w = uniform_i64(seed, 2, n, 0, 1_000_000, pinned=pinned)
    ref = GpuTableRef("memory", "main", table)
    return Workload("c0", c0_plan(v_lt, w_mod, ref),
                    [make_column("k", T.INT32, k), make_column("v", T.FLOAT64, v), make_column("w", T.INT64, w)],
                    n, 20.0, {"v_lt": v_lt, "w_mod": w_mod, "k_card": k_card}, {table: ["k", "v", "w"]})


def c1_plan(ts_gt: int, table: GpuTableRef | None = None) -> GpuPlanNode:
    scan = make_scan(["a", "b", "amt", "v", "ts"], table or GpuTableRef("memory", "main", "c1"))
    filt = make_filter([
        make_expr(f"((bool*)out)[idx] = (((const long long*)inputs[0])[row] > {int(ts_gt)}LL);", ["ts"], T.BOOLEAN),
    ], scan)
    return make_group_by(["a", "b"], [
        make_aggregate(A.SUM, "amt", T.HUGEINT),
        make_aggregate(A.AVG, "v", T.FLOAT64),
        make_aggregate(A.COUNT_STAR, "", T.INT64),
        make_aggregate(A.MAX, "ts", T.INT64),
    ], filt)


def c1(n: int = C1_ROWS, seed: int = 1, pinned: bool = False, table: str = "c1") -> Workload:
    a = zipf_i32(seed, 0, n, 1 << 20, 1.1, pinned=pinned)
    b = uniform_i32(seed, 1, n, 0, 16, pinned=pinned)
    amt = uniform_i64(seed, 2, n, 0, 1_000_000, pinned=pinned)
    v = uniform_f64(seed, 3, n, pinned=pinned)
    ts = uniform_i64(seed, 4, n, 0, 1 << 62, pinned=pinned)
    med = median_i64(ts)
    ref = GpuTableRef("memory", "main", table)
    return Workload("c1", c1_plan(med, ref),
                    [make_column("a", T.INT32, a), make_column("b", T.INT32, b), make_column("amt", T.INT64, amt),
                     make_column("v", T.FLOAT64, v), make_column("ts", T.INT64, ts)],
                    n, 32.0, {"ts_gt": med}, {table: ["a", "b", "amt", "v", "ts"]})


def c2_plan(probe: GpuTableRef | None = None, build: GpuTableRef | None = None) -> GpuPlanNode:
    left = make_scan(["pkey", "x"], probe or GpuTableRef("memory", "main", "c2_probe"))
    right = make_scan(["bkey", "g"], build or GpuTableRef("memory", "main", "c2_build"))
    join = make_join("pkey", "bkey", ["g", "x"], left, right)
    return make_group_by(["g"], [make_aggregate(A.SUM, "x", T.FLOAT64)], join)


def c2(probe_n: int = C2_PROBE_ROWS, build_n: int = C2_BUILD_ROWS, seed: int = 2, pinned: bool = False,
       miss_lo: int = 1 << 24, miss_span: int = 1 << 24) -> Workload:
    bkey = permutation_i64(seed, 0, build_n, pinned=pinned)
    g = uniform_i32(seed, 1, build_n, 0, 4096, pinned=pinned)
    cdf = zipf_cdf(build_n, 0.8)
    pkey = _alloc(probe_n, "<i8", pinned)
    datagen().vgdg_probe_keys_i64(seed, 2, 0, probe_n, bkey.ctypes.data, cdf.ctypes.data, build_n, 0.9,
                                  max(miss_lo, build_n), miss_span, pkey.ctypes.data)
    x = uniform_f64(seed, 3, probe_n, pinned=pinned)
    return Workload("c2", c2_plan(),
                    [make_column("pkey", T.INT64, pkey), make_column("x", T.FLOAT64, x),
                     make_column("bkey", T.INT64, bkey), make_column("g", T.INT32, g)],
                    probe_n, 16.0 + 12.0 * build_n / probe_n, {"build_n": build_n},
                    {"c2_probe": ["pkey", "x"], "c2_build": ["bkey", "g"]})


def c2b_plan(modulus: int = 13) -> GpuPlanNode:
    cross = make_cross_product(["a", "b"], make_scan(["a"], GpuTableRef("memory", "main", "c2b_l")),
                               make_scan(["b"], GpuTableRef("memory", "main", "c2b_r")))
    return make_filter([
        make_expr(f"((bool*)out)[idx] = (((((const int*)inputs[0])[row] + ((const int*)inputs[1])[row]) % "
                  f"{int(modulus)}) == 0);", ["a", "b"], T.BOOLEAN),
    ], cross)


def c2b(side: int = C2B_SIDE, seed: int = 5, modulus: int = 13) -> Workload:
    a = uniform_i32(seed, 0, side, 0, 1 << 20)
    b = uniform_i32(seed, 1, side, 0, 1 << 20)
    return Workload("c2b", c2b_plan(modulus), [make_column("a", T.INT32, a), make_column("b", T.INT32, b)],
                    side * side, 0.0, {"modulus": modulus, "side": side},
                    {"c2b_l": ["a"], "c2b_r": ["b"]})


C3_QUERIES = 256


def c3(n_queries: int = C3_QUERIES, seed: int = 3, min_log2: int = 10, max_log2: int = 22, card_lo: int = 16,
       card_hi: int = 1 << 16, pinned: bool = False) -> list[Workload]:
    """Batching workload: C0-shaped filter + group-by queries, each over its own table. Row counts are
    log-uniform over [2^min_log2, 2^max_log2], group cardinality log-uniform over [card_lo, card_hi];
    every query has its own predicate constants (v < v_lt, w % w_mod <> 0)."""
    rng = np.random.default_rng(seed)
    out = []
    for q in range(n_queries):
        n = int(round(2 ** rng.uniform(min_log2, max_log2)))
        k_card = int(round(2 ** rng.uniform(np.log2(card_lo), np.log2(card_hi))))
        v_lt = float(np.round(rng.uniform(0.1, 0.9), 6))
        w_mod = int(rng.integers(2, 17))
        wl = c0(n=n, seed=(seed << 16) + q, k_card=k_card, v_lt=v_lt, w_mod=w_mod, pinned=pinned, table=f"c3_q{q}")
        wl.name = "c3"
        out.append(wl)
    return out


def cp_plan(v_lt: float = 0.5, w_mod: int = 7, table: GpuTableRef | None = None) -> GpuPlanNode:
    """Filter + projection without the GROUP BY: SELECT k, v*2+1, w FROM t WHERE v<v_lt AND w%w_mod<>0."""
    return c0_plan(v_lt, w_mod, table).children[0]


def cp(n: int = C0_ROWS, seed: int = 0, pinned: bool = False, table: str = "c0") -> Workload:
    """The c0 table under its filter and projection alone (the fused FILTER/PROJECTION chain): 20 input
    bytes per row, and 20 bytes written per passing row (about 43% pass)."""
    wl = c0(n=n, seed=seed, pinned=pinned, table=table)
    wl.name = "cp"
    wl.plan = cp_plan(0.5, 7, GpuTableRef("memory", "main", table))
    return wl


def c2dup(probe_n: int = C2_PROBE_ROWS, build_n: int = C2_BUILD_ROWS, seed: int = 6, pinned: bool = False,
          repeat: int = 2) -> Workload:
    """The c2 join with a build side whose keys repeat: build_n rows holding build_n / repeat distinct keys
    (a seeded permutation, each key `repeat` times, in shuffled order) with their own g; probe keys drawn
    like c2's over the distinct keys (90% hits, Zipf(0.8) ranks; 10% misses). Every hit pairs with
    `repeat` build rows, so the join emits about 0.9 * repeat * probe_n pairs before the GROUP BY."""
    distinct = build_n // repeat
    keys = permutation_i64(seed, 0, distinct, pinned=False)
    order = permutation_i64(seed, 4, build_n, pinned=False)
    bkey = _alloc(build_n, "<i8", pinned)
    bkey[:] = np.tile(keys, repeat)[order]
    g = uniform_i32(seed, 1, build_n, 0, 4096, pinned=pinned)
    cdf = zipf_cdf(distinct, 0.8)
    pkey = _alloc(probe_n, "<i8", pinned)
    datagen().vgdg_probe_keys_i64(seed, 2, 0, probe_n, keys.ctypes.data, cdf.ctypes.data, distinct, 0.9,
                                  max(1 << 24, build_n), 1 << 24, pkey.ctypes.data)
    x = uniform_f64(seed, 3, probe_n, pinned=pinned)
    return Workload("c2dup", c2_plan(GpuTableRef("memory", "main", "c2dup_probe"),
                                     GpuTableRef("memory", "main", "c2dup_build")),
                    [make_column("pkey", T.INT64, pkey), make_column("x", T.FLOAT64, x),
                     make_column("bkey", T.INT64, bkey), make_column("g", T.INT32, g)],
                    probe_n, 16.0 + 12.0 * build_n / probe_n, {"build_n": build_n, "repeat": repeat},
                    {"c2dup_probe": ["pkey", "x"], "c2dup_build": ["bkey", "g"]})
