"""Row-range sharding of a group-by across ranks (one process per GPU, `torch.distributed`): each rank
runs the query on its own rows with the engine, and the partial groups are merged here.

`merge_dense_groupby` handles key domains small enough to index directly (the filter + group-by and
join + group-by shapes: at most 2^20 key values): every aggregate becomes a key-indexed array filled
with the rank's partial values (the identity elsewhere) and is combined with one all-reduce -- SUM
for sums and counts, MIN and MAX for those (in int64 over integer columns, in float64 with +-inf as
the identity over FLOAT32/FLOAT64 columns: kinds "min_f64"/"max_f64"). 128-bit integer sums (DuckDB's HUGEINT, the engine's
`{lower, upper}` pairs) travel as four 32-bit chunks summed in 64-bit lanes, which cannot overflow
for fewer than 2^31 ranks, and are carried back into 128 bits, so the merged sum is exact. AVG does
not merge from its outputs: shard its SUM and COUNT instead. `repartition_merge_groupby` handles key
spaces too large to index (the high-cardinality shape): partial groups move to the rank owning their
key's hash with all-to-all exchanges and merge there. Every rank makes the same collective calls in
the same order, whatever rows it holds (an empty partial contributes identities).

`sharded_group_by` runs a whole GROUP BY plan this way: it rewrites AVG into SUM + COUNT(*), runs the
plan on the rank's rows through a caller-supplied executor (the engine), packs multi-column keys from
their global ranges, picks one of the two merges by the packed domain, and finishes AVG exactly as the
engine's own finalize does.

Works with the "gloo" backend on CPU tensors and with "nccl" on CUDA tensors of the rank's device.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np

KINDS = ("sum_f64", "sum_i128", "count", "min", "max", "min_f64", "max_f64")
# MIN/MAX over integer columns merge as int64, over FLOAT32/FLOAT64 columns as float64 (identity +-inf)
_FLOAT_KINDS = ("sum_f64", "min_f64", "max_f64")
HUGEINT = np.dtype([("lower", "<u8"), ("upper", "<i8")])
_MAX_DOMAIN = 1 << 20


def _all_reduce(array: np.ndarray, op, device: str) -> np.ndarray:
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(np.ascontiguousarray(array)).to(device)
    dist.all_reduce(t, op=op)
    return t.cpu().numpy()


def merge_dense_groupby(keys: np.ndarray, aggregates: Sequence[tuple[str, np.ndarray]], key_min: int, key_max: int,
                        device: str = "cpu") -> tuple[np.ndarray, list[np.ndarray]]:
    """Merges this rank's partial groups (`keys`, one value per key and aggregate) with every other
    rank's. `key_min`/`key_max` bound the keys of all ranks (the same on every rank). Returns the
    merged keys in ascending order and the merged aggregates, the same on every rank."""
    import torch.distributed as dist
    keys = np.asarray(keys, dtype=np.int64)
    domain = int(key_max) - int(key_min) + 1
    if domain <= 0 or domain > _MAX_DOMAIN:
        raise ValueError(f"merge_dense_groupby: key domain of {domain} values is not dense (at most {_MAX_DOMAIN})")
    if keys.size and (keys.min() < key_min or keys.max() > key_max):
        raise ValueError("merge_dense_groupby: a key lies outside [key_min, key_max]")
    for kind, values in aggregates:  # checked before any collective, so every rank fails alike
        if kind not in KINDS:
            raise ValueError(f"merge_dense_groupby: aggregate kind {kind!r} does not merge (one of {KINDS})")
        if np.asarray(values).shape[0] != keys.shape[0]:
            raise ValueError("merge_dense_groupby: one value per key is needed")
    slot = keys - int(key_min)
    present = np.zeros(domain, np.int64)
    present[slot] = 1
    present = _all_reduce(present, dist.ReduceOp.SUM, device)
    live = np.nonzero(present)[0]
    merged = []
    for kind, values in aggregates:
        values = np.asarray(values)
        if kind == "sum_f64":
            dense = np.zeros(domain, np.float64)
            dense[slot] = values.astype(np.float64)
            merged.append(_all_reduce(dense, dist.ReduceOp.SUM, device)[live])
        elif kind == "count":
            dense = np.zeros(domain, np.int64)
            dense[slot] = values.astype(np.int64)
            merged.append(_all_reduce(dense, dist.ReduceOp.SUM, device)[live])
        elif kind in ("min", "max"):
            info = np.iinfo(np.int64)
            dense = np.full(domain, info.max if kind == "min" else info.min, np.int64)
            dense[slot] = values.astype(np.int64)
            op = dist.ReduceOp.MIN if kind == "min" else dist.ReduceOp.MAX
            merged.append(_all_reduce(dense, op, device)[live])
        elif kind in ("min_f64", "max_f64"):
            dense = np.full(domain, np.inf if kind == "min_f64" else -np.inf, np.float64)
            dense[slot] = values.astype(np.float64)
            op = dist.ReduceOp.MIN if kind == "min_f64" else dist.ReduceOp.MAX
            merged.append(_all_reduce(dense, op, device)[live])
        else:
            merged.append(_merge_i128(values, slot, domain, device)[live])
    return live.astype(np.int64) + int(key_min), merged


def _merge_i128(values: np.ndarray, slot: np.ndarray, domain: int, device: str) -> np.ndarray:
    """Exact sum over ranks of 128-bit integers given as {lower u64, upper i64}."""
    import torch.distributed as dist
    v = np.asarray(values).astype(HUGEINT, copy=False)
    lower = v["lower"].astype(np.uint64)
    upper = v["upper"].astype(np.int64)
    mask = np.uint64(0xFFFFFFFF)
    chunks = [  # value = c0 + c1 2^32 + c2 2^64 + c3 2^96, c0..c2 in [0, 2^32), c3 signed 32-bit
        (lower & mask).astype(np.int64),
        (lower >> np.uint64(32)).astype(np.int64),
        (upper.view(np.uint64) & mask).astype(np.int64),
        upper >> np.int64(32),
    ]
    sums = []
    for c in chunks:
        dense = np.zeros(domain, np.int64)
        dense[slot] = c
        sums.append(_all_reduce(dense, dist.ReduceOp.SUM, device))
    return _i128_from_chunks(sums)


def _owner(keys: np.ndarray, world: int) -> np.ndarray:
    """Rank owning each key: a 64-bit mix of the key (so skewed or sequential keys spread), mod world."""
    with np.errstate(over="ignore"):
        k = keys.astype(np.uint64)
        k = (k ^ (k >> np.uint64(33))) * np.uint64(0xFF51AFD7ED558CCD)
        k = (k ^ (k >> np.uint64(33))) * np.uint64(0xC4CEB9FE1A85EC53)
        k ^= k >> np.uint64(33)
    return (k % np.uint64(world)).astype(np.int64)


def _exchange(columns: list[np.ndarray], send_counts: np.ndarray, device: str) -> tuple[list[np.ndarray], np.ndarray]:
    """all_to_all of row-aligned int64/float64 columns already ordered by destination rank."""
    import torch
    import torch.distributed as dist
    world = send_counts.shape[0]
    recv_counts = torch.empty(world, dtype=torch.int64, device=device)
    dist.all_to_all_single(recv_counts, torch.from_numpy(send_counts.astype(np.int64)).to(device))
    recv = recv_counts.cpu().numpy()
    out = []
    for col in columns:
        src = torch.from_numpy(np.ascontiguousarray(col)).to(device)
        dst = torch.empty(int(recv.sum()), dtype=src.dtype, device=device)
        dist.all_to_all_single(dst, src, recv.tolist(), send_counts.tolist())
        out.append(dst.cpu().numpy())
    return out, recv


def _i128_from_chunks(chunk_sums: list[np.ndarray]) -> np.ndarray:
    """128-bit values from the sums of their 32-bit chunks (c0..c2 non-negative, c3 signed)."""
    low = []
    carry = np.zeros(chunk_sums[0].shape[0], np.int64)
    for s in chunk_sums[:3]:
        t = s + carry
        low.append((t & 0xFFFFFFFF).astype(np.uint64))
        carry = t >> 32
    top = chunk_sums[3] + carry
    out = np.empty(chunk_sums[0].shape[0], HUGEINT)
    out["lower"] = low[0] | (low[1] << np.uint64(32))
    out["upper"] = (low[2] | (top.view(np.uint64) << np.uint64(32))).view(np.int64)
    return out


def _i128_to_f64(values: np.ndarray) -> np.ndarray:
    """128-bit integers ({lower, upper}) to the nearest doubles (ties to even): values inside int64
    through numpy's int64 -> float64 conversion, which rounds that way; the rest through Python ints."""
    lower = values["lower"].astype(np.uint64)
    upper = values["upper"].astype(np.int64)
    small = ((upper == 0) & (lower < np.uint64(1 << 63))) | ((upper == -1) & (lower >= np.uint64(1 << 63)))
    out = lower.view(np.int64).astype(np.float64)
    for i in np.flatnonzero(~small).tolist():
        out[i] = float((int(upper[i]) << 64) | int(lower[i]))
    return out


def repartition_merge_groupby(keys: np.ndarray, aggregates: Sequence[tuple[str, np.ndarray]],
                              device: str = "cpu", reaggregate=None) -> tuple[np.ndarray, list[np.ndarray]]:
    """Merges partial groups of a key space too large to index (the high-cardinality shape): every
    partial group goes to the rank that owns its key (a hash of the key), with one all-to-all per
    column, and each rank merges what it received. `keys` are the packed group keys (int64). Returns
    this rank's share of the merged groups, keys ascending; the ranks' shares are disjoint and together
    hold every group. Exactness as in merge_dense_groupby.

    `reaggregate(plan, columns)`, when given, merges the received partials with a GROUP BY instead of
    numpy: the engine's, so the merge runs where the engine does (`lambda p, c:
    GpuEngine.instance().execute_plan(p, c).columns`). It gets a plan grouping INT64 column `k` with
    SUM (FP64 sums, and counts as 128-bit sums), MIN and MAX over the partial columns -- 128-bit sums
    as four 32-bit chunk columns whose exact sums are carried back into 128 bits, float MIN/MAX as
    order-preserving int64 words (the engine's MIN/MAX takes integer columns only) -- and returns the
    result columns (`.data`): key, then one per aggregate of the plan."""
    import torch.distributed as dist
    keys = np.asarray(keys, dtype=np.int64)
    for kind, values in aggregates:  # checked before any collective, so every rank fails alike
        if kind not in KINDS:
            raise ValueError(f"repartition_merge_groupby: aggregate kind {kind!r} does not merge (one of {KINDS})")
        if np.asarray(values).shape[0] != keys.shape[0]:
            raise ValueError("repartition_merge_groupby: one value per key is needed")
    world = dist.get_world_size()
    owner = _owner(keys, world)
    order = np.argsort(owner, kind="stable")
    send = np.bincount(owner, minlength=world).astype(np.int64)
    columns = [keys[order]]
    layout = []  # (kind, first column index, column count)
    for kind, values in aggregates:
        values = np.asarray(values)[order]
        if kind == "sum_i128":
            v = values.astype(HUGEINT, copy=False)
            layout.append((kind, len(columns), 2))
            columns += [v["lower"].view(np.int64), v["upper"].astype(np.int64)]
        else:
            layout.append((kind, len(columns), 1))
            columns.append(values.astype(np.float64 if kind in _FLOAT_KINDS else np.int64))
    got, _ = _exchange(columns, send, device)
    if reaggregate is not None:
        return _reaggregate(got, layout, reaggregate)
    rkeys = got[0]
    ukeys, pos = np.unique(rkeys, return_inverse=True)
    g = ukeys.shape[0]
    merged = []
    for kind, first, _n in layout:
        col = got[first]
        if kind == "sum_f64":
            acc = np.zeros(g, np.float64)
            np.add.at(acc, pos, col)
        elif kind == "count":
            acc = np.zeros(g, np.int64)
            np.add.at(acc, pos, col)
        elif kind in ("min", "max"):
            info = np.iinfo(np.int64)
            acc = np.full(g, info.max if kind == "min" else info.min, np.int64)
            (np.minimum if kind == "min" else np.maximum).at(acc, pos, col)
        elif kind in ("min_f64", "max_f64"):
            acc = np.full(g, np.inf if kind == "min_f64" else -np.inf, np.float64)
            (np.minimum if kind == "min_f64" else np.maximum).at(acc, pos, col)
        else:
            lower = col.view(np.uint64)
            upper = got[first + 1]
            mask = np.uint64(0xFFFFFFFF)
            chunks = [(lower & mask).astype(np.int64), (lower >> np.uint64(32)).astype(np.int64),
                      (upper.view(np.uint64) & mask).astype(np.int64), upper >> np.int64(32)]
            sums = []
            for c in chunks:  # at most 2^31 partials per group keep these sums inside 64 bits
                acc_c = np.zeros(g, np.int64)
                np.add.at(acc_c, pos, c)
                sums.append(acc_c)
            acc = _i128_from_chunks(sums)
        merged.append(acc)
    return ukeys, merged


def _f64_order_bits(values: np.ndarray) -> np.ndarray:
    """float64 values <-> int64 words whose signed order is the floats' order (NaN above +inf): the
    sign bit kept, the other 63 bits flipped for negative values. The map is its own inverse, so it
    also turns such words (given as int64) back into the float64 bit patterns."""
    b = np.ascontiguousarray(values).view(np.int64)
    return np.where(b < 0, b ^ np.int64(0x7FFFFFFFFFFFFFFF), b)


def _reaggregate(got: list[np.ndarray], layout, run) -> tuple[np.ndarray, list[np.ndarray]]:
    """The received partials merged by `run(plan, columns)` (a GROUP BY executor, see
    repartition_merge_groupby)."""
    from .engine import GpuAggregateKind as A, GpuValueType as T, make_aggregate, make_column, make_group_by, make_scan
    rows = got[0].shape[0]
    empty = {"sum_f64": np.float64, "count": np.int64, "min": np.int64, "max": np.int64, "sum_i128": HUGEINT,
             "min_f64": np.float64, "max_f64": np.float64}
    if rows == 0:  # nothing arrived: no executor call (no collective follows, so ranks stay in step)
        return np.zeros(0, np.int64), [np.zeros(0, empty[kind]) for kind, _, _ in layout]
    names, cols, aggs, slots = ["k"], [make_column("k", T.INT64, got[0])], [], []
    mask = np.uint64(0xFFFFFFFF)
    for i, (kind, first, _n) in enumerate(layout):
        if kind == "sum_i128":
            lower, upper = got[first].view(np.uint64), got[first + 1]
            parts = [(lower & mask).astype(np.int64), (lower >> np.uint64(32)).astype(np.int64),
                     (upper.view(np.uint64) & mask).astype(np.int64), upper >> np.int64(32)]
        else:
            parts = [got[first]]
        slots.append(len(aggs))
        for j, part in enumerate(parts):
            name = f"p{i}_{j}"
            names.append(name)
            if kind == "sum_f64":
                cols.append(make_column(name, T.FLOAT64, part))
                aggs.append(make_aggregate(A.SUM, name, T.FLOAT64))
            elif kind in ("min_f64", "max_f64"):  # as order-preserving int64 (the GPU MIN/MAX is integer-only)
                cols.append(make_column(name, T.INT64, _f64_order_bits(part)))
                aggs.append(make_aggregate(A.MIN if kind == "min_f64" else A.MAX, name, T.INT64))
            else:
                cols.append(make_column(name, T.INT64, part))
                agg = {"min": A.MIN, "max": A.MAX}.get(kind, A.SUM)
                aggs.append(make_aggregate(agg, name, T.HUGEINT if agg == A.SUM else T.INT64))
    out = [np.asarray(c.data) for c in run(make_group_by(["k"], aggs, make_scan(names)), cols)]
    if len(out) != 1 + len(aggs):
        raise ValueError("repartition_merge_groupby: the re-aggregation returned the wrong number of columns")
    order = np.argsort(out[0], kind="stable")
    ukeys = out[0][order].astype(np.int64)
    merged = []
    for (kind, _, _), at in zip(layout, slots):
        if kind == "sum_f64":
            merged.append(out[1 + at][order].astype(np.float64))
        elif kind in ("min_f64", "max_f64"):
            merged.append(_f64_order_bits(out[1 + at][order].astype(np.int64)).view(np.float64))
        elif kind in ("min", "max"):
            merged.append(out[1 + at][order].astype(np.int64))
        elif kind == "count":  # a 128-bit sum of counts: its low word
            merged.append(out[1 + at][order]["lower"].view(np.int64))
        else:  # four chunk sums, each below 2^63 for fewer than 2^31 partials per group
            merged.append(_i128_from_chunks([out[1 + at + j][order]["lower"].view(np.int64) for j in range(4)]))
    return ukeys, merged


def _partial_plan(node, column_types, who: str):
    """The GROUP BY `node` rewritten to partial states that merge: AVG as SUM (HUGEINT over integers,
    DOUBLE over floats, per `column_types`) plus one shared COUNT(*). Returns (plan, merge kinds,
    finish steps, index of the shared count or None)."""
    from .engine import GpuAggregateKind as A, GpuOpType, GpuPlanNode, GpuValueType as T, make_aggregate
    if node.op_type != GpuOpType.GROUP_BY_AGGREGATE or not node.group_keys:
        raise ValueError(f"{who}: a GROUP BY node with group keys is needed")
    column_types = dict(column_types or {})
    plan_aggs, kinds, finish = [], [], []
    count_at = None
    for a in node.aggregates:
        if a.kind == A.AVG:
            if a.input_column not in column_types:
                raise ValueError(f"{who}: the value type of AVG input {a.input_column!r} is needed")
            is_float = T(column_types[a.input_column]) in (T.FLOAT32, T.FLOAT64)
            s = len(plan_aggs)
            plan_aggs.append(make_aggregate(A.SUM, a.input_column, T.FLOAT64 if is_float else T.HUGEINT))
            kinds.append("sum_f64" if is_float else "sum_i128")
            if count_at is None:
                count_at = len(plan_aggs)
                plan_aggs.append(make_aggregate(A.COUNT_STAR, "", T.INT64))
                kinds.append("count")
            finish.append(("avg", s, is_float))
        else:
            out_t = T(a.output_type)
            finish.append(("col", len(plan_aggs), out_t))
            plan_aggs.append(a)
            if a.kind in (A.COUNT_STAR, A.COUNT):
                kinds.append("count")
            elif a.kind in (A.MIN, A.MAX):
                suffix = "_f64" if out_t in (T.FLOAT32, T.FLOAT64) else ""
                kinds.append(("min" if a.kind == A.MIN else "max") + suffix)
            else:
                kinds.append("sum_i128" if out_t == T.HUGEINT else "sum_f64")
    plan = GpuPlanNode(node.op_type, list(node.children), estimated_rows=node.estimated_rows,
                       estimated_row_width_bytes=node.estimated_row_width_bytes, group_keys=list(node.group_keys),
                       aggregates=plan_aggs)
    return plan, kinds, finish, count_at


def sharded_group_by(node, run_local, column_types=None, device: str = "cpu", reaggregate=None):
    """A GROUP BY over rows split across ranks. `run_local(plan)` runs `plan` on this rank's rows (with
    the engine, say `lambda p: GpuEngine.instance().execute_plan(p, my_inputs).columns`) and returns its
    host result columns (GpuColumn-like: `.data` and `.validity`; the group keys, then one column per
    aggregate). AVG runs as SUM plus COUNT(*) -- `column_types` maps each AVG input to its value type,
    which decides the SUM: HUGEINT over integers, DOUBLE over floats -- and is finished after the merge
    as the engine finishes it (the 128-bit sum correctly rounded to double, then divided by the group's
    row count). Keys pack like the engine's: each key column offset by its global minimum (found with
    an all-reduce) in as many bits as its global range needs. A packed domain of at most 2^20 values
    merges densely and every rank gets the whole result; a larger one merges by hash repartition and
    each rank gets a disjoint share. Groups come sorted by their keys, first key first. Dictionary-string
    keys must use one dictionary on every rank. NULL group keys or NULL aggregate outputs are refused on
    every rank alike. `reaggregate` is passed to repartition_merge_groupby. Returns
    [(name, numpy array)]: the keys by name, then `agg_<i>` per aggregate of `node`, in order."""
    import torch.distributed as dist
    from .engine import GpuValueType as T, NUMPY_DTYPE
    plan, kinds, finish, count_at = _partial_plan(node, column_types, "sharded_group_by")
    plan_aggs = plan.aggregates
    cols = list(run_local(plan))
    nk = len(node.group_keys)
    if len(cols) != nk + len(plan_aggs):
        raise ValueError("sharded_group_by: the local result has the wrong number of columns")
    nulls = any(c.validity is not None and not np.all(c.validity) for c in cols)
    keys = [np.asarray(c.data).astype(np.int64) for c in cols[:nk]]
    key_dtypes = [np.asarray(c.data).dtype for c in cols[:nk]]
    rows = keys[0].shape[0]
    info = np.iinfo(np.int64)
    lo = _all_reduce(np.array([k.min() if rows else info.max for k in keys], np.int64), dist.ReduceOp.MIN, device)
    hi = _all_reduce(np.array([k.max() if rows else info.min for k in keys] + [int(nulls)], np.int64),
                     dist.ReduceOp.MAX, device)
    if hi[-1]:
        raise ValueError("sharded_group_by: NULL group keys or NULL aggregate values do not merge here")
    hi = hi[:-1]
    empty = lo[0] > hi[0]  # no rank has a group
    bits = [0] * nk if empty else [int(h - l).bit_length() for l, h in zip(lo.tolist(), hi.tolist())]
    if sum(bits) > 63:
        raise ValueError("sharded_group_by: the group keys need more than 63 bits packed")
    shifts = [sum(bits[i + 1:]) for i in range(nk)]  # first key highest: ascending packed = lexicographic
    aggs = list(zip(kinds, [c.data for c in cols[nk:]]))
    if empty:
        mkeys = np.zeros(0, np.int64)
        merged = [np.zeros(0, HUGEINT if k == "sum_i128" else np.float64 if k in _FLOAT_KINDS else np.int64)
                  for k in kinds]
    else:
        packed = np.zeros(rows, np.int64)
        for k, l, sh in zip(keys, lo.tolist(), shifts):
            packed |= (k - l) << sh
        if (1 << sum(bits)) <= _MAX_DOMAIN:
            mkeys, merged = merge_dense_groupby(packed, aggs, 0, (1 << sum(bits)) - 1, device)
        else:
            mkeys, merged = repartition_merge_groupby(packed, aggs, device, reaggregate)
    out = []
    for name, l, b, sh, dt in zip(node.group_keys, lo.tolist(), bits, shifts, key_dtypes):
        out.append((name, (((mkeys >> sh) & ((1 << b) - 1)) + l).astype(dt)))
    for i, f in enumerate(finish):
        if f[0] == "avg":
            _, s, is_float = f
            n = merged[count_at]
            if is_float:
                vals = merged[s] / n.astype(np.float64)
            else:
                vals = _i128_to_f64(merged[s]) / n.astype(np.float64)
        else:
            _, s, t = f
            vals = merged[s] if t in (T.HUGEINT, T.FLOAT64) else merged[s].astype(NUMPY_DTYPE[t])
        out.append((f"agg_{i}", vals))
    return out


def _raw_column(result, i: int):
    """The vgpu_column of a device result (its device data and validity pointers)."""
    import ctypes as C
    from . import abi
    c = abi.vgpu_column()
    abi.check(abi.lib().vgpu_result_get_column(result._handle, i, C.byref(c)))
    return c


_TORCH_KEY_DTYPE = {"BOOLEAN": "uint8", "INT16": "int16", "INT32": "int32", "INT64": "int64", "DICTIONARY_STRING": "int32"}


def device_sharded_group_by(node, inputs, column_types=None):
    """A GROUP BY over rows split across ranks, merged on the GPUs: the device counterpart of
    sharded_group_by for the nccl backend (one process per GPU, torch's current device and stream).

    The plan runs on this rank's `inputs` with the engine, results left on the device (partial states:
    AVG as SUM + COUNT(*), as in sharded_group_by). The key ranges meet in two small all-reduces; every
    partial group is then packed into one row of 64-bit words and routed to the rank owning its key
    (vgpu_shard_route), the rows cross the ranks in one all-to-all of device buffers, become columns
    again (vgpu_shard_columns), are re-aggregated by the engine's GROUP BY on the owning rank, and the
    output columns are built on the device (vgpu_shard_finish). Nothing passes through the host but the
    per-rank row counts and the key ranges.

    Returns [(name, torch tensor on this rank's device)]: the keys by name, then `agg_<i>` per aggregate
    of `node` (HUGEINT as an (n, 2) int64 tensor of {lower, upper}). This rank holds a disjoint share of
    the groups, in no particular order; the shares of all ranks hold every group once. Exactness as
    sharded_group_by (FP64 sums merged in an order that depends on the exchange). Every rank makes the
    same collective calls in the same order; NULL keys or partial states are refused on every rank."""
    import torch
    import torch.distributed as dist
    plan, kinds, finish, count_at = _partial_plan(node, column_types, "device_sharded_group_by")
    world = dist.get_world_size()
    dev = torch.device("cuda", torch.cuda.current_device())
    # Everything -- engine calls, shard kernels, torch allocations and the NCCL exchange -- is ordered on
    # one stream the engine can be handed (not the legacy default stream, which the engine's own stream
    # does not wait on).
    caller = torch.cuda.current_stream()
    side = caller if caller.cuda_stream != 0 else torch.cuda.Stream()
    side.wait_stream(caller)
    with torch.cuda.stream(side):
        out = _device_sharded_group_by_on(node, inputs, plan, kinds, finish, count_at, world, dev, side.cuda_stream)
    if side is not caller:
        caller.wait_stream(side)
        for _, t in out:
            t.record_stream(caller)
    return out


def _device_sharded_group_by_on(node, inputs, plan, kinds, finish, count_at, world, dev, sp):
    import torch
    import torch.distributed as dist
    from .engine import (DeviceResult, ExecuteOptions, GpuAggregateKind as A, GpuEngine, GpuValueType as T,
                         make_aggregate, make_device_column, make_group_by, make_scan)
    opts = ExecuteOptions(output_on_device=True, stream=sp)
    eng = GpuEngine.instance()
    nk = len(node.group_keys)
    held = []

    def run(p, cols):
        r = eng.execute_plan(p, cols, opts)
        if not isinstance(r, DeviceResult):
            raise RuntimeError(f"device_sharded_group_by: {r.error_message}")
        held.append(r)
        return r

    try:
        local = run(plan, inputs)
        raw = [_raw_column(local, i) for i in range(len(local.columns))]
        if len(raw) != nk + len(plan.aggregates):
            raise ValueError("device_sharded_group_by: the local result has the wrong number of columns")
        rows = int(raw[0].row_count)
        key_types = [T(c.type) for c in raw[:nk]]
        nulls = any(bool(c.validity) for c in raw)
        info = np.iinfo(np.int64)
        lo_l, hi_l = [info.max] * nk, [info.min] * nk
        if rows:  # local key ranges: the engine's MIN/MAX without group keys over the key columns
            names = [f"k{j}" for j in range(nk)]
            aggs = [make_aggregate(kd, n, t) for n, t in zip(names, key_types) for kd in (A.MIN, A.MAX)]
            mm = eng.execute_plan(make_group_by([], aggs, make_scan(names)),
                                  [make_device_column(n, t, int(c.data), rows) for n, t, c in zip(names, key_types, raw)],
                                  ExecuteOptions(stream=sp))
            if not mm.success:
                raise RuntimeError(f"device_sharded_group_by: {mm.error_message}")
            lo_l = [int(mm.columns[2 * j].data[0]) for j in range(nk)]
            hi_l = [int(mm.columns[2 * j + 1].data[0]) for j in range(nk)]
        lo = _all_reduce(np.array(lo_l, np.int64), dist.ReduceOp.MIN, dev)
        hi = _all_reduce(np.array(hi_l + [int(nulls)], np.int64), dist.ReduceOp.MAX, dev)
        if hi[-1]:
            raise ValueError("device_sharded_group_by: NULL group keys or NULL aggregate values do not merge here")
        hi = hi[:-1]
        empty = bool(lo[0] > hi[0])
        bits = [0] * nk if empty else [int(h - l).bit_length() for l, h in zip(lo.tolist(), hi.tolist())]
        if sum(bits) > 63:
            raise ValueError("device_sharded_group_by: the group keys need more than 63 bits packed")
        shifts = [sum(bits[i + 1:]) for i in range(nk)]
        send, send_splits = _route_partials(raw, nk, kinds, [int(x) for x in lo.tolist()], shifts, world, sp)
        recv = exchange_rows(send, send_splits)
        del send
        return _merge_exchanged(recv, kinds, finish, count_at, list(node.group_keys), key_types, shifts, bits,
                                [int(x) for x in lo.tolist()], run, sp)
    finally:
        for r in held:  # frees on the stream the work was queued on, after it
            r.free()


def exchange_rows(send, send_splits):
    """The all-to-all of routed rows: `send` is a (rows, words) int64 tensor on this rank's device (CUDA
    with nccl, CPU with gloo) whose first send_splits[0] rows go to rank 0, the next send_splits[1] to
    rank 1, and so on. The row counts cross first (one all-to-all of `world` int64), then the rows (one
    all-to-all). Returns the received rows, sender by sender, as a (received rows, words) tensor."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size()
    if len(send_splits) != world or sum(send_splits) != int(send.shape[0]):
        raise ValueError("exchange_rows: one row count per rank, summing to the rows sent")
    dev = send.device
    recv_counts = torch.empty(world, dtype=torch.int64, device=dev)
    dist.all_to_all_single(recv_counts, torch.tensor(list(send_splits), dtype=torch.int64, device=dev))
    recv_splits = recv_counts.cpu().tolist()
    recv = torch.empty((int(sum(recv_splits)), int(send.shape[1])), dtype=torch.int64, device=dev)
    dist.all_to_all_single(recv, send, recv_splits, list(send_splits))
    return recv


def _route_partials(raw, nk: int, kinds, lo, shifts, world: int, stream: int):
    """vgpu_shard_route over a device result's columns (nk keys, then the partial states): the rows as
    an int64 (rows, words) tensor grouped by owner rank, and the rows per rank (host list)."""
    import ctypes as C
    import torch
    from . import abi
    L = abi.lib()
    rows = int(raw[0].row_count)
    codes = [KINDS.index(k) for k in kinds]
    kinds_c = (C.c_int32 * max(1, len(codes)))(*codes)
    words = int(L.vgpu_shard_words(kinds_c, len(codes)))
    send = torch.empty((rows, words), dtype=torch.int64, device=torch.device("cuda", torch.cuda.current_device()))
    counts = (C.c_uint64 * world)()
    abi.check(L.vgpu_shard_route((abi.vgpu_column * nk)(*raw[:nk]), nk, (C.c_int64 * nk)(*lo), (C.c_int32 * nk)(*shifts),
                                 (abi.vgpu_column * max(1, len(codes)))(*raw[nk:]), kinds_c, len(codes), rows, world,
                                 C.c_void_p(send.data_ptr() if rows else 0), counts, C.c_void_p(stream)))
    return send, [int(x) for x in counts]


def _merge_exchanged(recv, kinds, finish, count_at, key_names, key_types, shifts, bits, lo, run, stream: int):
    """Received partial-group rows (int64 (R, words) device tensor) re-aggregated by the engine's GROUP
    BY (`run(plan, columns)` returns a device result it keeps alive) and finished into the query's output
    columns: [(name, tensor)] as device_sharded_group_by returns them."""
    import ctypes as C
    import torch
    from . import abi
    from .engine import GpuAggregateKind as A, GpuValueType as T, make_aggregate, make_device_column, make_group_by, make_scan
    L = abi.lib()
    dev = recv.device
    R, W = int(recv.shape[0]), int(recv.shape[1])
    nk = len(key_names)
    out_names = list(key_names) + [f"agg_{i}" for i in range(len(finish))]
    if R == 0:  # nothing arrived: no engine call (no collective follows, so ranks stay in step)
        return _empty_device_outputs(out_names, key_types, finish, kinds, dev)
    cols = torch.empty((W, R), dtype=torch.int64, device=dev)
    abi.check(L.vgpu_shard_columns(C.c_void_p(recv.data_ptr()), R, W, C.c_void_p(cols.data_ptr()), C.c_void_p(stream)))
    names, dcols, aggs, at = ["k"], [make_device_column("k", T.INT64, cols[0].data_ptr(), R)], [], []
    w = 1
    for kind in kinds:
        at.append(len(aggs))
        for _ in range(4 if kind == "sum_i128" else 1):
            name = f"w{w}"
            names.append(name)
            if kind == "sum_f64":
                dcols.append(make_device_column(name, T.FLOAT64, cols[w].data_ptr(), R))
                aggs.append(make_aggregate(A.SUM, name, T.FLOAT64))
            else:
                dcols.append(make_device_column(name, T.INT64, cols[w].data_ptr(), R))
                if kind in ("min", "max", "min_f64", "max_f64"):
                    aggs.append(make_aggregate(A.MIN if kind.startswith("min") else A.MAX, name, T.INT64))
                else:
                    aggs.append(make_aggregate(A.SUM, name, T.HUGEINT))
            w += 1
    merged = run(make_group_by(["k"], aggs, make_scan(names)), dcols)
    mraw = [_raw_column(merged, i) for i in range(len(merged.columns))]
    G = int(mraw[0].row_count)
    outs, tensors = [], []

    def output(op, dst, srcs=(), count=None, key=None):
        o = abi.vgpu_shard_output()
        o.op = op
        for j, c in enumerate(srcs):
            o.src[j] = c
        if count is not None:
            o.count = count
        if key is not None:
            o.key_type, o.key_shift, o.key_bits, o.key_min = key
        o.dst = dst.data_ptr()
        outs.append(o)
        tensors.append(dst)

    for j in range(nk):
        t = torch.empty(G, dtype=getattr(torch, _TORCH_KEY_DTYPE[key_types[j].name]), device=dev)
        output(abi.SHARD_OUT_KEY, t, [mraw[0]], key=(int(key_types[j]), shifts[j], bits[j], int(lo[j])))
    count_col = mraw[1 + at[count_at]] if count_at is not None else None
    for f in finish:
        s = f[1]
        src = mraw[1 + at[s]: 1 + at[s] + (4 if kinds[s] == "sum_i128" else 1)]
        if f[0] == "avg":
            op = abi.SHARD_OUT_AVG_F64 if f[2] else abi.SHARD_OUT_AVG_I128
            output(op, torch.empty(G, dtype=torch.float64, device=dev), src, count=count_col)
        elif kinds[s] == "sum_i128":
            output(abi.SHARD_OUT_I128, torch.empty((G, 2), dtype=torch.int64, device=dev), src)
        elif kinds[s] in ("min_f64", "max_f64"):
            output(abi.SHARD_OUT_F64_FROM_ORDER, torch.empty(G, dtype=torch.float64, device=dev), src)
        elif kinds[s] == "sum_f64":
            output(abi.SHARD_OUT_WORD, torch.empty(G, dtype=torch.float64, device=dev), src)
        else:
            output(abi.SHARD_OUT_WORD, torch.empty(G, dtype=torch.int64, device=dev), src)
    abi.check(L.vgpu_shard_finish((abi.vgpu_shard_output * len(outs))(*outs), len(outs), G, C.c_void_p(stream)))
    result = []
    for name, t, f in zip(out_names, tensors, [None] * nk + list(finish)):
        if f is not None and f[0] == "col" and kinds[f[1]] in ("count", "min", "max", "min_f64", "max_f64"):
            want = _torch_dtype_of(f[2])
            if want is not None and t.dtype != want:
                t = t.to(want)
        result.append((name, t))
    return result


def _torch_dtype_of(t):
    import torch
    return {"INT16": torch.int16, "INT32": torch.int32, "INT64": torch.int64, "FLOAT32": torch.float32,
            "FLOAT64": torch.float64, "BOOLEAN": torch.uint8}.get(t.name)


def _empty_device_outputs(names, key_types, finish, kinds, dev):
    """The outputs of a rank that received no groups (the same names, dtypes and shapes, no rows)."""
    import torch
    out = [(name, torch.empty(0, dtype=getattr(torch, _TORCH_KEY_DTYPE[t.name]), device=dev))
           for name, t in zip(names, key_types)]
    for i, f in enumerate(finish):
        if f[0] == "avg":
            t = torch.empty(0, dtype=torch.float64, device=dev)
        elif kinds[f[1]] == "sum_i128":
            t = torch.empty((0, 2), dtype=torch.int64, device=dev)
        else:
            t = torch.empty(0, dtype=_torch_dtype_of(f[2]) or torch.int64, device=dev)
        out.append((f"agg_{i}", t))
    return out


def broadcast_table(columns, src: int = 0, device: str = "cpu") -> dict:
    """The join + group-by shape sharded by probe rows needs the whole build side on every rank: rank
    `src` passes its columns ({name: 1-D numpy array}, any fixed-width dtype including HUGEINT), the
    others pass None, and every rank returns the same columns. Names, dtypes and lengths travel first
    (one object broadcast), then each column as its raw bytes (one broadcast per column)."""
    import torch
    import torch.distributed as dist
    if dist.get_rank() == src:
        cols = {name: np.ascontiguousarray(np.asarray(v)) for name, v in columns.items()}
        if any(v.ndim != 1 or v.dtype.hasobject for v in cols.values()):
            header = [None]  # refused on every rank after the header broadcast
        else:
            header = [[(name, v.dtype.descr if v.dtype.names else v.dtype.str, v.shape[0])
                       for name, v in cols.items()]]
    else:
        cols, header = None, [None]
    dist.broadcast_object_list(header, src=src)
    if header[0] is None:
        raise ValueError("broadcast_table: columns must be 1-D arrays of a fixed-width dtype")
    out = {}
    for name, descr, rows in header[0]:
        dtype = np.dtype([tuple(f) for f in descr]) if isinstance(descr, list) else np.dtype(descr)
        if cols is not None:
            buf = torch.from_numpy(cols[name].view(np.uint8).copy()).to(device)
        else:
            buf = torch.empty(rows * dtype.itemsize, dtype=torch.uint8, device=device)
        dist.broadcast(buf, src=src)
        out[name] = buf.cpu().numpy().view(dtype)
    return out
