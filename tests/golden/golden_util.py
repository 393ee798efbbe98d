"""Canonical form and comparison of operator results against the golden fixtures.

A result is a list of columns; it is turned into rows (NULL cells as None unless the fixture checks
stored values under NULLs), ordered per the fixture's comparison (positional, group set sorted by the
key columns, or row multiset sorted by all columns). Large expected results are stored as a SHA-256
digest of the canonical JSON rows plus their count.
"""
from __future__ import annotations

import hashlib
import json
import math

import numpy as np

FULL_LIMIT = 2000  # cells; above this the fixture stores a digest


def _cell(v):
    if isinstance(v, (np.floating, float)):
        f = float(v)
        return 0.0 if f == 0.0 else f
    if isinstance(v, np.void):  # HUGEINT
        return int(v["upper"]) * (1 << 64) + int(v["lower"])
    if isinstance(v, (np.integer, int, bool, np.bool_)):
        return int(v)
    return v


def result_rows(columns, null_values_checked: bool) -> tuple[list[list], list[list[int]]]:
    """columns: objects with .data (numpy) and .validity (bool array or None)."""
    n = len(columns[0].data) if columns else 0
    rows = [[None] * len(columns) for _ in range(n)]
    nulls = []
    for j, c in enumerate(columns):
        vals = [_cell(x) for x in c.data]
        valid = c.validity if c.validity is not None else None
        for i in range(n):
            if valid is not None and not valid[i]:
                nulls.append([i, j])
                rows[i][j] = vals[i] if null_values_checked else None
            else:
                rows[i][j] = vals[i]
    return rows, nulls


def canonical(rows: list[list], compare: str, keys: int) -> list[list]:
    def key_all(r):
        return [(x is None, x if x is not None else 0) for x in r]
    if compare == "ordered":
        return rows
    if compare == "set":
        return sorted(rows, key=lambda r: key_all(r[:keys]) if keys else 0)
    if compare == "multiset":
        return sorted(rows, key=key_all)
    raise ValueError(compare)


def digest(rows: list[list]) -> str:
    return hashlib.sha256(json.dumps(rows, separators=(",", ":")).encode()).hexdigest()


def encode_expected(exp: dict) -> dict:
    """Turns a case expectation into the stored fixture (full rows or digest)."""
    if not exp["success"]:
        return exp
    out = dict(exp)
    rows = canonical([[_cell(x) for x in r] for r in exp["rows"]], exp["compare"], exp["keys"])
    nulls = exp.get("nulls", [])
    if not exp.get("null_values_checked"):
        for i, j in nulls:
            if exp["compare"] == "ordered":
                rows[i][j] = None
    cells = sum(len(r) for r in rows)
    out.pop("rows")
    if cells <= FULL_LIMIT:
        out["rows"] = rows
    else:
        out["digest"] = digest(rows)
        out["head"] = rows[:5]
    out["nulls"] = nulls
    return out


def check(fixture: dict, success: bool, error: str, columns) -> str | None:
    """Returns None when the result matches the fixture, else a description of the mismatch."""
    if not fixture["success"]:
        if success:
            return "expected a refusal, got success"
        if fixture.get("error_contains") and fixture["error_contains"] not in error:
            return f"refusal message {error!r} lacks {fixture['error_contains']!r}"
        return None
    if not success:
        return f"expected success, got error: {error}"
    rows, nulls = result_rows(columns, fixture.get("null_values_checked", False))
    if len(rows) != fixture["row_count"]:
        return f"row count {len(rows)} != {fixture['row_count']}"
    if fixture["compare"] == "ordered" and sorted(nulls) != sorted(fixture.get("nulls", [])):
        return f"NULL cells {nulls[:10]} != {fixture.get('nulls', [])[:10]}"
    rows = canonical(rows, fixture["compare"], fixture["keys"])
    if fixture["compare"] == "set" and fixture["keys"]:
        ks = [tuple(r[:fixture["keys"]]) for r in rows]
        if len(set(ks)) != len(ks):
            return "duplicate group keys"
    if "digest" in fixture:
        d = digest(rows)
        if d != fixture["digest"]:
            return f"digest mismatch (head {rows[:3]} vs {fixture['head'][:3]})"
        return None
    tol = fixture.get("float_tol", 0.0)
    for i, (a, b) in enumerate(zip(rows, fixture["rows"])):
        for x, y in zip(a, b):
            if isinstance(y, float) and isinstance(x, (int, float)) and x is not None:
                if not (x == y or (tol and abs(x - y) <= tol) or (math.isnan(x) and math.isnan(y))):
                    return f"row {i}: {a} != {b}"
            elif x != y:
                return f"row {i}: {a} != {b}"
    return None
