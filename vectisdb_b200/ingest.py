"""The host ingest path over the C ABI: DuckDB-shaped vectors (UnifiedVectorFormat: physical values,
selection vector, validity mask words, constant flag) converted like the reference extension's
vector_converter (extension/src/vector_converter.cpp:87-273) and accumulated into page-locked batches
that are uploaded asynchronously into the device column cache (gpu_batch_accumulator.cpp:126-249 plus
the scan's upload, re-built around overlapped transfers).

    with TableIngest(GpuTableRef("memory", "main", "t"), [("k", T.INT32), ("v", T.FLOAT64)]) as ing:
        for chunk in scan:                       # 2048-row chunks
            ing.append([Vector(k_data), Vector(v_data, validity=mask)], len(chunk))
    # the table is committed to the column cache when the block ends
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import abi
from .engine import GpuTableRef, GpuValueType, NUMPY_DTYPE


@dataclass
class Vector:
    """One vector of a chunk: `data` the physical values (numpy), `sel` the logical -> physical selection
    (uint32, optional), `validity` DuckDB's mask words by physical index (uint64, LSB first, bit set =
    valid; optional), `constant` every logical row reads physical value 0."""
    data: np.ndarray
    sel: np.ndarray | None = None
    validity: np.ndarray | None = None
    constant: bool = False


def _c_vector(v: Vector, keep: list) -> abi.vgpu_vector:
    data = np.ascontiguousarray(v.data)
    keep.append(data)
    out = abi.vgpu_vector()
    out.data = data.ctypes.data
    if v.sel is not None:
        sel = np.ascontiguousarray(v.sel, dtype=np.uint32)
        keep.append(sel)
        out.sel = sel.ctypes.data_as(C.POINTER(C.c_uint32))
    if v.validity is not None:
        val = np.ascontiguousarray(v.validity, dtype=np.uint64)
        keep.append(val)
        out.validity = val.ctypes.data_as(C.POINTER(C.c_uint64))
    out.constant = 1 if v.constant else 0
    return out


def _c_sel(row_sel, keep: list):
    if row_sel is None:
        return None
    sel = np.ascontiguousarray(row_sel, dtype=np.uint32)
    keep.append(sel)
    return sel.ctypes.data_as(C.POINTER(C.c_uint32))


def convert_vector(v: Vector, t: GpuValueType, count: int, row_sel=None):
    """ConvertVectorToGpuColumn: (dense values, Arrow validity bitmap or None when no row is NULL)."""
    keep: list = []
    cv = _c_vector(v, keep)
    out = np.empty(count, dtype=NUMPY_DTYPE[GpuValueType(t)])
    bitmap = np.empty((count + 7) // 8, dtype=np.uint8)
    any_null = C.c_int()
    abi.check(abi.lib().vgpu_convert_vector(C.byref(cv), int(t), count, _c_sel(row_sel, keep), out.ctypes.data,
                                            bitmap.ctypes.data, C.byref(any_null)))
    return out, (bitmap if any_null.value else None)


def validity_words(valid: np.ndarray) -> np.ndarray:
    """A boolean per-row validity array as DuckDB's 64-bit mask words (LSB first)."""
    valid = np.asarray(valid, dtype=bool)
    padded = np.zeros((len(valid) + 63) // 64 * 64, dtype=bool)
    padded[: len(valid)] = valid
    return np.packbits(padded, bitorder="little").view(np.uint64)


class TableIngest:
    """vgpu_ingest_*: appended chunks staged into the column cache table `table`; `finish()` (or leaving
    a `with` block normally) commits, a handle dropped unfinished aborts."""

    def __init__(self, table: GpuTableRef, columns: Sequence[tuple[str, GpuValueType]], batch_rows: int = 1 << 20):
        self._keep = [abi.vgpu_table_ref(table.catalog.encode(), table.schema.encode(), table.table.encode())]
        names = (C.c_char_p * len(columns))(*[n.encode() for n, _ in columns])
        types = (C.c_int32 * len(columns))(*[int(t) for _, t in columns])
        self._keep += [names, types]
        self.types = [GpuValueType(t) for _, t in columns]
        self._h = C.c_void_p()
        abi.check(abi.lib().vgpu_ingest_create(C.byref(self._keep[0]), names, types, len(columns), batch_rows,
                                               C.byref(self._h)))

    def append(self, vectors: Sequence[Vector], count: int, row_sel=None) -> None:
        keep: list = []
        arr = (abi.vgpu_vector * len(vectors))(*[_c_vector(v, keep) for v in vectors])
        abi.check(abi.lib().vgpu_ingest_append(self._h, arr, count, _c_sel(row_sel, keep)))

    def finish(self) -> int:
        rows = C.c_uint64()
        abi.check(abi.lib().vgpu_ingest_finish(self._h, C.byref(rows)))
        return int(rows.value)

    def close(self) -> None:
        if self._h:
            abi.lib().vgpu_ingest_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, exc_type, *exc):
        try:
            if exc_type is None:
                self.finish()
        finally:
            self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
