"""Bound expressions -> engine expressions (the reference extension's TranslateExpression and
WrapAsOutputStatement, extension/src/expression_translator.cpp:287-460, 489-493, over the C ABI's
vgpu_translate_expression).

A bound expression tree is built from the four classes DuckDB's binder produces -- `col` (a bound
column reference), `const` (a bound constant), `cmp` (a bound comparison) and `fn` (a bound function,
by DuckDB's function name: "+", "-", "*", "/", "%", "__cast", "abs", "sqrt", "ln", ...) -- each with its
return type, and `translate` returns the GpuExpr the engine's plans carry: the statement
`((T*)out)[idx] = ...;`, the input columns in slot order and the output type.

    v_lt = cmp("<", col("v", T.FLOAT64), const(0.5, T.FLOAT64))
    expr = translate(v_lt)   # ((bool*)out)[idx] = (((const double*)inputs[0])[row] < 0.5);
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

from . import abi
from .engine import GpuExpr, GpuValueType

COLUMN, CONSTANT, COMPARE, FUNCTION = 0, 1, 2, 3
FP32 = 1        # VECTOR_GPU_FP32_RELAXATION: math functions in float
STRICT_FP = 2   # VECTOR_GPU_STRICT_FP: only the bit-exact math functions


@dataclass
class BoundExpr:
    kind: int
    return_type: GpuValueType
    name: str = ""
    children: list = field(default_factory=list)
    value: object = None  # constants; None = NULL


def col(name: str, t: GpuValueType) -> BoundExpr:
    return BoundExpr(COLUMN, GpuValueType(t), name)


def const(value, t: GpuValueType) -> BoundExpr:
    return BoundExpr(CONSTANT, GpuValueType(t), value=value)


def cmp(op: str, left: BoundExpr, right: BoundExpr) -> BoundExpr:
    return BoundExpr(COMPARE, GpuValueType.BOOLEAN, op, [left, right])


def fn(name: str, t: GpuValueType, *args: BoundExpr) -> BoundExpr:
    return BoundExpr(FUNCTION, GpuValueType(t), name, list(args))


def cast(x: BoundExpr, t: GpuValueType) -> BoundExpr:
    return fn("__cast", t, x)


def _flatten(root: BoundExpr):
    nodes, keep = [], []

    def add(e: BoundExpr) -> int:
        idx = len(nodes)
        nodes.append(None)
        kids = [add(c) for c in e.children]
        arr = (C.c_uint32 * max(1, len(kids)))(*kids)
        keep.append(arr)
        name = e.name.encode() if e.name else None
        keep.append(name)
        b = abi.vgpu_bexpr(kind=e.kind, return_type=int(e.return_type), name=name,
                           children=C.cast(arr, C.POINTER(C.c_uint32)), n_children=len(kids),
                           is_null=1 if (e.kind == CONSTANT and e.value is None) else 0)
        if e.kind == CONSTANT and e.value is not None:
            if e.return_type in (GpuValueType.FLOAT32, GpuValueType.FLOAT64):
                b.f64 = float(e.value)
            else:
                b.i64 = int(e.value)
        nodes[idx] = b
        return idx

    add(root)
    return (abi.vgpu_bexpr * len(nodes))(*nodes), keep


def translate(root: BoundExpr, flags: int = 0) -> GpuExpr:
    """The engine expression for `root`; raises abi.VgpuError(VGPU_ERR_UNSUPPORTED) with the reason for
    shapes the GPU path does not lower (the caller falls back to DuckDB's CPU path)."""
    arr, _keep = _flatten(root)
    cap = 1 << 16
    stmt = C.create_string_buffer(cap)
    names = C.create_string_buffer(cap)
    slen, nlen = C.c_size_t(), C.c_size_t()
    n_in, out_t = C.c_uint32(), C.c_uint32()
    abi.check(abi.lib().vgpu_translate_expression(arr, len(arr), 0, flags, stmt, cap, C.byref(slen), names, cap,
                                                  C.byref(nlen), C.byref(n_in), C.byref(out_t)))
    inputs = [s.decode() for s in names.raw[:nlen.value].split(b"\0")[:n_in.value]]
    return GpuExpr(stmt.value.decode(), inputs, GpuValueType(out_t.value))
