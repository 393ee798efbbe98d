"""Plan-level CPU oracle (TEST INFRASTRUCTURE ONLY): evaluates a GpuPlanNode over host columns with the
reference engine's semantics, operator by operator, at sizes that finish in seconds.

    SCAN        inputs consumed positionally in traversal order, names from the inputs
                (cuda_engine/src/gpu_executor.cu:531-560); NULLs refused unless the plan is
                row-independent (gpu_executor_internal.hpp: ExecContext::nulls_supported)
    FILTER      AND of all predicates, a NULL predicate excludes the row, child columns compacted in
                order (gpu_executor.cu:645-730)
    PROJECTION  one output col<i> per expression, NULL iff any referenced input is NULL
                (gpu_executor.cu:279-323, code_generator.cpp:269-310)
    GROUP BY    type/shape checks and messages of operators/gpu_groupby.cu:224-350; groups ordered
                by key tuple; DOUBLE sums accumulated in row order; integer SUM exact (HUGEINT)
    HASH_JOIN   one equality key, same integer type both sides, every left row paired with its
                matching right rows (operators/gpu_hash_join.cu:138-267)
    CROSS       left-major pairs (operators/gpu_cross_join.cu:111-192)

Expressions are the reference's own CUDA statements compiled as C by gcc (-ffp-contract=off), each
wrapped in a dense loop exactly like the reference's fused kernel body.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from vectisdb_b200.engine import (GpuAggregateKind as A, GpuOpType as Op, GpuPlanNode, GpuValueType as T,
                                  NUMPY_DTYPE)

HERE = Path(__file__).resolve().parent
EXPR_DIR = HERE / "_build" / "expr"

_PRELUDE = """#include <stdbool.h>
#include <math.h>
static inline double __vgpu_radians(double d) { return d * 0.017453292519943295; }
static inline double __vgpu_degrees(double r) { return r * 57.29577951308232; }
void vgpu_oracle_expr(const void **inputs, void *out, unsigned long long n) {
  for (unsigned long long idx = 0; idx < n; idx++) {
    const unsigned long long row = idx; (void)row;
    %s
  }
}
"""

_EXPR_CACHE: dict = {}


class OracleRefusal(Exception):
    """The reference engine refuses this plan (message mirrors its error text)."""


def _compile(source: str):
    if source in _EXPR_CACHE:
        return _EXPR_CACHE[source]
    code = _PRELUDE % source
    h = hashlib.sha256(code.encode()).hexdigest()[:24]
    EXPR_DIR.mkdir(parents=True, exist_ok=True)
    so = EXPR_DIR / f"e_{h}.so"
    if not so.exists():
        c = EXPR_DIR / f"e_{h}.c"
        c.write_text(code)
        subprocess.run(["gcc", "-O1", "-ffp-contract=off", "-fPIC", "-shared", "-o", str(so), str(c), "-lm"],
                       check=True, capture_output=True)
    lib = C.CDLL(str(so))
    fn = lib.vgpu_oracle_expr
    fn.argtypes = [C.POINTER(C.c_void_p), C.c_void_p, C.c_ulonglong]
    fn.restype = None
    _EXPR_CACHE[source] = (lib, fn)
    return lib, fn


@dataclass
class Col:
    name: str
    type: T
    data: np.ndarray
    valid: np.ndarray | None = None  # bool per row or None

    @property
    def rows(self) -> int:
        return len(self.data)


def eval_expr(expr, cols: list[Col], rows: int) -> Col:
    srcs = []
    valid = None
    for name in expr.input_columns:
        c = _find(cols, name, "gpu_executor: input column")
        if c.rows != rows:
            raise OracleRefusal(f"gpu_executor: input column '{name}' row count mismatch")
        srcs.append(np.ascontiguousarray(c.data))
        if c.valid is not None:
            valid = c.valid.copy() if valid is None else (valid & c.valid)
    out = np.zeros(rows, dtype=NUMPY_DTYPE[expr.output_type])
    if rows:
        _, fn = _compile(expr.generated_cuda_source)
        arr = (C.c_void_p * max(1, len(srcs)))(*[s.ctypes.data for s in srcs])
        fn(arr, out.ctypes.data, rows)
    return Col("", expr.output_type, out, valid)


def _find(cols: list[Col], name: str, what: str) -> Col:
    for c in cols:
        if c.name == name:
            return c
    raise OracleRefusal(f"{what} '{name}' not found")


def _row_independent(node: GpuPlanNode) -> bool:
    if node.op_type == Op.SCAN:
        return True
    if node.op_type in (Op.FILTER, Op.PROJECTION):
        return all(_row_independent(c) for c in node.children)
    return False


class PlanOracle:
    def __init__(self, inputs):
        self.inputs = inputs
        self.cursor = 0
        self.nulls_ok = True

    def run(self, plan: GpuPlanNode) -> list[Col]:
        self.nulls_ok = _row_independent(plan)
        return self.exec(plan)

    def exec(self, n: GpuPlanNode) -> list[Col]:
        return {Op.SCAN: self.scan, Op.FILTER: self.filter, Op.PROJECTION: self.projection,
                Op.GROUP_BY_AGGREGATE: self.group_by, Op.HASH_JOIN: self.join,
                Op.CROSS_PRODUCT: self.cross}[n.op_type](n)

    def scan(self, n):
        out = []
        for _ in n.column_names:
            if self.cursor >= len(self.inputs):
                raise OracleRefusal("gpu_executor: plan expects more scanned columns than were supplied")
            g = self.inputs[self.cursor]
            self.cursor += 1
            if g.validity is not None and not self.nulls_ok:
                raise OracleRefusal(f"gpu_executor: column '{g.name}' contains NULLs, which this operator does not model")
            out.append(Col(g.name, g.type, np.asarray(g.data, dtype=NUMPY_DTYPE[g.type]),
                           None if g.validity is None else np.asarray(g.validity, bool)))
        return out

    def filter(self, n):
        if len(n.children) != 1:
            raise OracleRefusal("gpu_executor: FILTER expects exactly one child")
        cols = self.exec(n.children[0])
        if not cols:
            return cols
        rows = cols[0].rows
        if not n.expressions or rows == 0:
            return cols
        mask = np.ones(rows, bool)
        for e in n.expressions:
            if e.output_type != T.BOOLEAN:
                raise OracleRefusal("gpu_executor: FILTER predicate did not evaluate to BOOLEAN")
            r = eval_expr(e, cols, rows)
            mask &= r.data.astype(bool)
            if r.valid is not None:
                mask &= r.valid
        return [Col(c.name, c.type, c.data[mask], None if c.valid is None else c.valid[mask]) for c in cols]

    def projection(self, n):
        if len(n.children) != 1:
            raise OracleRefusal("gpu_executor: PROJECTION expects exactly one child")
        cols = self.exec(n.children[0])
        rows = cols[0].rows if cols else 0
        out = []
        for i, e in enumerate(n.expressions):
            r = eval_expr(e, cols, rows)
            r.name = f"col{i}"
            out.append(r)
        return out

    def group_by(self, n):
        if len(n.children) != 1:
            raise OracleRefusal("gpu_executor: GROUP_BY_AGGREGATE expects exactly one child")
        cols = self.exec(n.children[0])
        if not cols:
            raise OracleRefusal("gpu_groupby: input operator produced no columns to group")
        if not n.group_keys and not n.aggregates:
            raise OracleRefusal("gpu_groupby: node has neither group keys nor aggregates")
        rows = cols[0].rows
        keys = []
        for k in n.group_keys:
            c = _find(cols, k, "gpu_groupby: group key column")
            if c.type not in (T.INT16, T.INT32, T.INT64, T.BOOLEAN):
                raise OracleRefusal(f"gpu_groupby: group key '{k}' is not an integer/boolean column, which this "
                                    f"GPU path requires")
            keys.append(c)
        for a in n.aggregates:
            if a.kind == A.COUNT_STAR:
                if a.output_type != T.INT64:
                    raise OracleRefusal("gpu_groupby: COUNT(*) must produce INT64")
                continue
            c = _find(cols, a.input_column, "gpu_groupby: aggregate input column")
            if a.kind == A.COUNT and a.output_type != T.INT64:
                raise OracleRefusal("gpu_groupby: COUNT must produce INT64")
            if a.kind == A.SUM:
                if c.type in (T.FLOAT32, T.FLOAT64):
                    if a.output_type != T.FLOAT64:
                        raise OracleRefusal("gpu_groupby: SUM on this GPU path supports only FLOAT/DOUBLE input "
                                            "producing DOUBLE")
                elif c.type in (T.INT16, T.INT32, T.INT64):
                    if a.output_type != T.HUGEINT:
                        raise OracleRefusal("gpu_groupby: SUM over an integer column must produce HUGEINT")
                else:
                    raise OracleRefusal("gpu_groupby: SUM on this GPU path supports only FLOAT/DOUBLE input "
                                        "producing DOUBLE")
            if a.kind == A.AVG:
                if a.output_type != T.FLOAT64:
                    raise OracleRefusal("gpu_groupby: AVG must produce DOUBLE")
                if c.type not in (T.INT16, T.INT32, T.INT64, T.FLOAT32, T.FLOAT64):
                    raise OracleRefusal("gpu_groupby: AVG supports numeric columns only")
            if a.kind in (A.MIN, A.MAX):
                if a.output_type != c.type:
                    raise OracleRefusal("gpu_groupby: MIN/MAX output type must match its input column type")
                if c.type not in (T.INT16, T.INT32, T.INT64, T.BOOLEAN):
                    raise OracleRefusal("gpu_groupby: MIN/MAX on this GPU path supports only integer/boolean columns")
        if rows == 0:
            if not n.group_keys:
                raise OracleRefusal("gpu_groupby: global aggregate over an empty input needs NULL results, which "
                                    "this GPU path cannot represent")
            return ([Col(k, c.type, np.zeros(0, NUMPY_DTYPE[c.type])) for k, c in zip(n.group_keys, keys)] +
                    [Col(f"agg_{i}", a.output_type, np.zeros(0, NUMPY_DTYPE[a.output_type]))
                     for i, a in enumerate(n.aggregates)])
        # group ids by lexicographic key order (stable: rows keep their order inside a group)
        if keys:
            order = np.lexsort([k.data.astype(np.int64) for k in reversed(keys)])
            sorted_keys = [k.data[order] for k in keys]
            head = np.ones(rows, bool)
            head[1:] = False
            for sk in sorted_keys:
                head[1:] |= sk[1:] != sk[:-1]
            gid_sorted = np.cumsum(head) - 1
            gid = np.empty(rows, np.int64)
            gid[order] = gid_sorted
            ngroups = int(gid_sorted[-1]) + 1
            reps = order[head]
        else:
            gid = np.zeros(rows, np.int64)
            ngroups = 1
            reps = np.zeros(1, np.int64)
        out = [Col(name, k.type, k.data[reps]) for name, k in zip(n.group_keys, keys)]
        counts = np.bincount(gid, minlength=ngroups).astype(np.int64)
        for i, a in enumerate(n.aggregates):
            name = f"agg_{i}"
            if a.kind in (A.COUNT_STAR, A.COUNT):
                out.append(Col(name, T.INT64, counts.copy()))
                continue
            c = _find(cols, a.input_column, "")
            vals = c.data
            if a.kind in (A.SUM, A.AVG):
                if c.type in (T.FLOAT32, T.FLOAT64):
                    s = np.zeros(ngroups, np.float64)
                    np.add.at(s, gid, vals.astype(np.float64))  # sequential, row order
                    res = s if a.kind == A.SUM else s / counts
                    out.append(Col(name, T.FLOAT64, res))
                else:
                    exact = [0] * ngroups
                    for g_, x in zip(gid.tolist(), vals.astype(np.int64).tolist()):
                        exact[g_] += x
                    if a.kind == A.AVG:
                        out.append(Col(name, T.FLOAT64, np.array([float(s) / cnt for s, cnt in
                                                                  zip(exact, counts.tolist())], np.float64)))
                    else:
                        h = np.zeros(ngroups, dtype=NUMPY_DTYPE[T.HUGEINT])
                        for j, s in enumerate(exact):
                            u = s & ((1 << 128) - 1)
                            h[j]["lower"] = u & ((1 << 64) - 1)
                            h[j]["upper"] = np.int64(np.uint64(u >> 64).astype(np.int64))
                        out.append(Col(name, T.HUGEINT, h))
            elif a.kind in (A.MIN, A.MAX):
                v64 = vals.astype(np.int64)
                r = np.full(ngroups, np.iinfo(np.int64).max if a.kind == A.MIN else np.iinfo(np.int64).min, np.int64)
                (np.minimum if a.kind == A.MIN else np.maximum).at(r, gid, v64)
                out.append(Col(name, c.type, r.astype(NUMPY_DTYPE[c.type])))
        return out

    def _resolve_side(self, name, left, right, op):
        lc = [c for c in left if c.name == name]
        rc = [c for c in right if c.name == name]
        if lc and rc:
            raise OracleRefusal(f"{op}: output column '{name}' is ambiguous (present on both sides)")
        if not lc and not rc:
            raise OracleRefusal(f"{op}: output column '{name}' not found on either side")
        return (lc[0], True) if lc else (rc[0], False)

    def join(self, n):
        if len(n.children) != 2:
            raise OracleRefusal("gpu_executor: HASH_JOIN expects exactly two children")
        left = self.exec(n.children[0])
        right = self.exec(n.children[1])
        if len(n.build_keys) != 1 or len(n.probe_keys) != 1:
            raise OracleRefusal("gpu_hash_join: this GPU path joins on exactly one equality key column")
        if not n.output_columns:
            raise OracleRefusal("gpu_hash_join: node has no output columns")
        lk = _find(left, n.build_keys[0], "gpu_hash_join: left key column")
        rk = _find(right, n.probe_keys[0], "gpu_hash_join: right key column")
        for side, k in (("left", lk), ("right", rk)):
            if k.type not in (T.INT16, T.INT32, T.INT64, T.BOOLEAN):
                raise OracleRefusal(f"gpu_hash_join: {side} join key is not an integer/boolean column, which this "
                                    f"GPU path requires")
        if lk.type != rk.type:
            raise OracleRefusal("gpu_hash_join: join key columns must have the same type on both sides")
        srcs = [self._resolve_side(nm, left, right, "gpu_hash_join") for nm in n.output_columns]
        order = np.argsort(rk.data, kind="stable")
        sk = rk.data[order]
        lo = np.searchsorted(sk, lk.data, "left")
        hi = np.searchsorted(sk, lk.data, "right")
        cnt = hi - lo
        li = np.repeat(np.arange(lk.rows), cnt)
        starts = np.repeat(lo, cnt)
        offs = np.arange(len(li)) - np.repeat(np.cumsum(cnt) - cnt, cnt)
        ri = order[starts + offs] if len(li) else np.zeros(0, np.int64)
        return [Col(nm, c.type, c.data[li] if is_left else c.data[ri])
                for nm, (c, is_left) in zip(n.output_columns, srcs)]

    def cross(self, n):
        if len(n.children) != 2:
            raise OracleRefusal("gpu_executor: CROSS_PRODUCT expects exactly two children")
        if not n.output_columns:
            raise OracleRefusal("gpu_cross_join: node has no output columns")
        left = self.exec(n.children[0])
        right = self.exec(n.children[1])
        srcs = [self._resolve_side(nm, left, right, "gpu_cross_join") for nm in n.output_columns]
        ln, rn = left[0].rows, right[0].rows
        if ln and rn and ln * rn > (1 << 32):
            raise OracleRefusal(f"gpu_cross_join: cross product of {ln} x {rn} rows is too large for GPU execution")
        li = np.repeat(np.arange(ln), rn)
        ri = np.tile(np.arange(rn), ln)
        return [Col(nm, c.type, c.data[li] if is_left else c.data[ri]) for nm, (c, is_left) in zip(n.output_columns, srcs)]


def evaluate(plan: GpuPlanNode, inputs) -> list[Col]:
    """Raises OracleRefusal where the reference engine refuses the plan."""
    return PlanOracle(list(inputs)).run(plan)
