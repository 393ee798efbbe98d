"""Sharded GROUP BY (vectisdb_b200.distributed.sharded_group_by): two gloo ranks on the CPU each run the
query on their own rows, through a numpy stand-in for the engine that does what the engine's group-by
returns (keys, then one column per aggregate; AVG must arrive rewritten as SUM + COUNT(*)). The merged
result must equal the same GROUP BY over all rows: exactly for keys, counts, MIN/MAX, 128-bit sums and
integer AVG (the 128-bit sum is exact however the rows are split, so its correctly rounded quotient is
too), within 1e-12 relative for FP64 sums and float AVG. Covered: two key columns in a dense packed
domain (every rank gets the whole result), a sparse 40-bit key (hash repartition, disjoint shares), a
rank with no rows, no rows anywhere, a join + group-by whose build side is broadcast from one rank
while the probe rows are split, and NULL keys refused on both ranks without a hang."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from vectisdb_b200.engine import (GpuAggregateKind as A, GpuColumn, GpuValueType as T, HUGEINT_DTYPE,  # noqa: E402
                                  make_aggregate, make_group_by, make_join, make_scan)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _exact_sums(values, pos, groups):
    """Exact per-group sums of int64 values as Python ints (32-bit halves summed in int64 lanes)."""
    v = values.astype(np.int64)
    lo = (v & 0xFFFFFFFF).astype(np.int64)
    hi = v >> 32
    slo = np.zeros(groups, np.int64)
    shi = np.zeros(groups, np.int64)
    np.add.at(slo, pos, lo)
    np.add.at(shi, pos, hi)
    return [(int(h) << 32) + int(l) for h, l in zip(shi.tolist(), slo.tolist())]


def _group(plan, arrays, allow_avg, validity=None):
    """The GROUP BY of `plan` over `arrays`, as the engine returns it (GpuColumn per output)."""
    keys = [np.asarray(arrays[k]) for k in plan.group_keys]
    n = keys[0].shape[0]
    if n:
        uniq, pos = np.unique(np.stack([k.astype(np.int64) for k in keys], 1), axis=0, return_inverse=True)
        pos = pos.reshape(-1)
    else:
        uniq, pos = np.zeros((0, len(keys)), np.int64), np.zeros(0, np.int64)
    g = uniq.shape[0]
    cnt = np.bincount(pos, minlength=g).astype(np.int64)
    cols = [GpuColumn(name, T.INT64, uniq[:, i].astype(keys[i].dtype)) for i, name in enumerate(plan.group_keys)]
    if validity is not None:
        cols[0].validity = validity(g)
    for a in plan.aggregates:
        x = None if a.kind == A.COUNT_STAR else np.asarray(arrays[a.input_column])
        if a.kind == A.COUNT_STAR:
            vals = cnt
        elif a.kind == A.SUM and a.output_type == T.FLOAT64:
            vals = np.zeros(g)
            np.add.at(vals, pos, x)
        elif a.kind == A.SUM:
            vals = np.zeros(g, HUGEINT_DTYPE)
            for i, t in enumerate(_exact_sums(x, pos, g)):
                vals[i]["lower"] = t & ((1 << 64) - 1)
                u = (t >> 64) & ((1 << 64) - 1)
                vals[i]["upper"] = u - (1 << 64) if u >= 1 << 63 else u
        elif a.kind in (A.MIN, A.MAX):
            info = np.finfo(x.dtype) if x.dtype.kind == "f" else np.iinfo(x.dtype)
            vals = np.full(g, info.max if a.kind == A.MIN else info.min, x.dtype)
            (np.minimum if a.kind == A.MIN else np.maximum).at(vals, pos, x)
        elif a.kind == A.AVG and allow_avg:
            if x.dtype.kind == "f":
                s = np.zeros(g)
                np.add.at(s, pos, x)
                vals = s / cnt
            else:
                vals = np.array([float(t) / float(c) for t, c in zip(_exact_sums(x, pos, g), cnt.tolist())])
        else:
            raise AssertionError(f"the local plan must not carry aggregate {a.kind!r}")
        cols.append(GpuColumn(f"agg", a.output_type, vals))
    return cols


def _dense_case(seed):
    rng = np.random.default_rng(seed)
    n = 20000
    arrays = {
        "g1": rng.integers(-3, 13, n).astype(np.int32),
        "g2": rng.integers(0, 41, n).astype(np.int16),
        "x": rng.random(n) + 1.0,
        "v": rng.integers((1 << 62) - 1000, 1 << 62, n, dtype=np.int64) * rng.choice([-1, 1], n),
        "w": rng.integers(-(1 << 40), 1 << 40, n, dtype=np.int64),
    }
    node = make_group_by(["g1", "g2"], [
        make_aggregate(A.COUNT_STAR, "", T.INT64), make_aggregate(A.SUM, "x", T.FLOAT64),
        make_aggregate(A.AVG, "v", T.FLOAT64), make_aggregate(A.MIN, "w", T.INT64),
        make_aggregate(A.MAX, "w", T.INT64), make_aggregate(A.AVG, "x", T.FLOAT64),
        make_aggregate(A.SUM, "v", T.HUGEINT)], make_scan(list(arrays)))
    return node, arrays


def _sparse_case(seed):
    rng = np.random.default_rng(seed)
    n = 60000
    k = rng.integers(0, 1 << 40, 30000)[rng.integers(0, 30000, n)]
    k[rng.random(n) < 0.1] = 12345  # a heavy key
    arrays = {"k": k.astype(np.int64),
              "v": rng.integers((1 << 62) - 1000, 1 << 62, n, dtype=np.int64) * rng.choice([-1, 1], n)}
    node = make_group_by(["k"], [make_aggregate(A.AVG, "v", T.FLOAT64), make_aggregate(A.SUM, "v", T.HUGEINT),
                                 make_aggregate(A.COUNT_STAR, "", T.INT64)], make_scan(list(arrays)))
    return node, arrays


def _float_minmax_case(seed, sparse):
    """MIN/MAX over DOUBLE and FLOAT columns with negative and fractional values (they must merge as
    floats, not be truncated to integers), beside SUM and COUNT(*); dense or sparse 40-bit keys."""
    rng = np.random.default_rng(seed)
    n = 30000
    if sparse:
        k = rng.integers(0, 1 << 40, 20000)[rng.integers(0, 20000, n)].astype(np.int64)
    else:
        k = rng.integers(-7, 60, n).astype(np.int32)
    arrays = {"k": k, "d": rng.standard_normal(n) * 1e3 - 0.25,
              "f": (rng.standard_normal(n) * 7.5).astype(np.float32)}
    node = make_group_by(["k"], [make_aggregate(A.MIN, "d", T.FLOAT64), make_aggregate(A.MAX, "d", T.FLOAT64),
                                 make_aggregate(A.MIN, "f", T.FLOAT32), make_aggregate(A.MAX, "f", T.FLOAT32),
                                 make_aggregate(A.COUNT_STAR, "", T.INT64), make_aggregate(A.SUM, "d", T.FLOAT64)],
                         make_scan(list(arrays)))
    return node, arrays


def _join_case(seed):
    """A key/foreign-key join feeding a group-by on a build-side column (the join + group-by shape)."""
    rng = np.random.default_rng(seed)
    nb, n = 4096, 30000
    build = {"bk": rng.permutation(nb).astype(np.int32), "bv": rng.integers(0, 300, nb).astype(np.int16),
             "bh": np.zeros(nb, HUGEINT_DTYPE)}
    build["bh"]["lower"] = rng.integers(0, 1 << 63, nb, dtype=np.int64).astype(np.uint64)
    build["bh"]["upper"] = rng.integers(-5, 5, nb)
    probe = {"pk": rng.integers(0, nb + 200, n).astype(np.int32),  # some probe keys miss
             "x": rng.random(n) + 1.0,
             "v": rng.integers((1 << 62) - 1000, 1 << 62, n, dtype=np.int64) * rng.choice([-1, 1], n)}
    node = make_group_by(["bv"], [make_aggregate(A.COUNT_STAR, "", T.INT64), make_aggregate(A.AVG, "v", T.FLOAT64),
                                  make_aggregate(A.SUM, "x", T.FLOAT64), make_aggregate(A.AVG, "x", T.FLOAT64)],
                         make_join("bk", "pk", ["bv", "x", "v"], make_scan(["bk", "bv"]), make_scan(["pk", "x", "v"])))
    return node, build, probe


def _join(build, probe):
    """Inner join of probe rows with the unique build keys: the probe rows that match, with bv."""
    order = np.argsort(build["bk"])
    sk = build["bk"][order]
    pos = np.minimum(np.searchsorted(sk, probe["pk"]), len(sk) - 1)
    hit = sk[pos] == probe["pk"]
    out = {k: v[hit] for k, v in probe.items()}
    out["bv"] = build["bv"][order][pos[hit]]
    return out


TYPES = {"x": T.FLOAT64, "v": T.INT64}


def _slice(arrays, lo, hi):
    return {k: v[lo:hi] for k, v in arrays.items()}


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    from vectisdb_b200.distributed import sharded_group_by
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        node, arrays = _dense_case(3)
        n = len(arrays["g1"])
        part = _slice(arrays, 0, n // 3) if rank == 0 else _slice(arrays, n // 3, n)
        out[("dense", rank)] = sharded_group_by(node, lambda p: _group(p, part, False), TYPES)
        part = arrays if rank == 0 else _slice(arrays, 0, 0)  # rank 1 holds no rows
        out[("one_empty", rank)] = sharded_group_by(node, lambda p: _group(p, part, False), TYPES)
        part = _slice(arrays, 0, 0)
        out[("all_empty", rank)] = sharded_group_by(node, lambda p: _group(p, part, False), TYPES)
        node, arrays = _sparse_case(4)
        n = len(arrays["k"])
        part = _slice(arrays, 0, n // 2) if rank == 0 else _slice(arrays, n // 2, n)
        out[("sparse", rank)] = sharded_group_by(node, lambda p: _group(p, part, False), TYPES)
        for sparse in (False, True):
            node, arrays = _float_minmax_case(8, sparse)
            n = len(arrays["k"])
            part = _slice(arrays, 0, n // 3) if rank == 0 else _slice(arrays, n // 3, n)
            out[("float_minmax", sparse, rank)] = sharded_group_by(node, lambda p: _group(p, part, False), TYPES)
        node, build, probe = _join_case(6)
        from vectisdb_b200.distributed import broadcast_table
        got = broadcast_table(build if rank == 0 else None)
        out[("broadcast", rank)] = got
        n = len(probe["pk"])
        part = _slice(probe, 0, n // 4) if rank == 0 else _slice(probe, n // 4, n)
        out[("join", rank)] = sharded_group_by(node, lambda p: _group(p, _join(got, part), False), TYPES)
        try:  # a column that is not fixed-width: refused on both ranks, after the one header broadcast
            broadcast_table({"names": np.array(["a", "b"], dtype=object)} if rank == 0 else None)
            out[("bad_broadcast", rank)] = "sent"
        except ValueError as e:
            out[("bad_broadcast", rank)] = str(e)
        node, arrays = _dense_case(5)
        validity = (lambda g: np.arange(g) != 0) if rank == 1 else None  # one NULL key on rank 1 only
        try:
            sharded_group_by(node, lambda p: _group(p, arrays, False, validity), TYPES)
            out[("nulls", rank)] = "merged"
        except ValueError as e:
            out[("nulls", rank)] = str(e)
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module")
def results():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    return dict(out)


def _expect(node, arrays):
    cols = _group(node, arrays, True)
    return [(name, c.data) for name, c in zip(list(node.group_keys) + [f"agg_{i}" for i in range(len(node.aggregates))],
                                              cols)]


def _check(got, exp, node):
    assert [n for n, _ in got] == [n for n, _ in exp]
    nk = len(node.group_keys)
    for (name, g), (_, e), i in zip(got, exp, range(len(exp))):
        a = node.aggregates[i - nk] if i >= nk else None
        if a is not None and a.kind in (A.MIN, A.MAX):  # MIN/MAX of any type: bit-exact, its own dtype
            assert g.dtype == e.dtype and np.array_equal(g, e), name
        elif a is not None and a.output_type == T.FLOAT64 and not (a.kind == A.AVG and a.input_column == "v"):
            assert g.dtype == np.float64
            assert np.all(np.abs(g - e) <= 1e-12 * np.abs(e)), name
        elif a is not None and a.output_type == T.HUGEINT:
            assert np.array_equal(g["lower"], e["lower"]) and np.array_equal(g["upper"], e["upper"]), name
        else:  # keys (their own dtype), counts, MIN/MAX and integer AVG: bit-exact
            assert g.dtype == e.dtype and np.array_equal(g, e), name


def test_dense_keys_merge_to_the_whole_result_on_every_rank(results):
    node, arrays = _dense_case(3)
    exp = _expect(node, arrays)
    for rank in (0, 1):
        _check(results[("dense", rank)], exp, node)
        _check(results[("one_empty", rank)], exp, node)


def test_no_rows_anywhere_gives_typed_empty_columns(results):
    node, _ = _dense_case(3)
    for rank in (0, 1):
        got = dict(results[("all_empty", rank)])
        assert got["g1"].dtype == np.int32 and got["g2"].dtype == np.int16 and len(got["g1"]) == 0
        assert got["agg_0"].dtype == np.int64 and got["agg_2"].dtype == np.float64
        assert got["agg_6"].dtype == HUGEINT_DTYPE and all(len(v) == 0 for v in got.values())


def test_sparse_keys_repartition_into_disjoint_shares(results):
    node, arrays = _sparse_case(4)
    exp = _expect(node, arrays)
    a, b = results[("sparse", 0)], results[("sparse", 1)]
    assert len(a[0][1]) > 0 and len(b[0][1]) > 0
    assert len(np.intersect1d(a[0][1], b[0][1])) == 0
    order = np.argsort(np.concatenate([a[0][1], b[0][1]]))
    got = [(na, np.concatenate([va, vb])[order]) for (na, va), (_, vb) in zip(a, b)]
    _check(got, exp, node)


def test_float_min_max_merge_as_floats(results):
    """MIN/MAX over DOUBLE/FLOAT keep their fractional and negative values and their dtype through the
    dense merge (every rank gets the whole result) and the hash repartition (disjoint shares)."""
    node, arrays = _float_minmax_case(8, False)
    exp = _expect(node, arrays)
    assert np.any(exp[1][1] != np.round(exp[1][1])) and np.any(exp[1][1] < 0)
    for rank in (0, 1):
        _check(results[("float_minmax", False, rank)], exp, node)
    node, arrays = _float_minmax_case(8, True)
    exp = _expect(node, arrays)
    a, b = results[("float_minmax", True, 0)], results[("float_minmax", True, 1)]
    assert len(a[0][1]) > 0 and len(b[0][1]) > 0 and len(np.intersect1d(a[0][1], b[0][1])) == 0
    order = np.argsort(np.concatenate([a[0][1], b[0][1]]))
    _check([(na, np.concatenate([va, vb])[order]) for (na, va), (_, vb) in zip(a, b)], exp, node)


def test_broadcast_build_side_and_probe_sharded_join_group_by(results):
    node, build, probe = _join_case(6)
    for rank in (0, 1):
        got = results[("broadcast", rank)]
        assert list(got) == list(build)
        for name in build:
            assert got[name].dtype == build[name].dtype and got[name].tobytes() == build[name].tobytes()
        _check(results[("join", rank)], _expect(node, _join(build, probe)), node)


def test_broadcast_refuses_object_columns_on_both_ranks(results):
    for rank in (0, 1):
        assert "fixed-width" in results[("bad_broadcast", rank)]


def test_null_keys_are_refused_on_both_ranks(results):
    for rank in (0, 1):
        assert "NULL" in results[("nulls", rank)]


def test_refusals_before_any_collective():
    """No process group exists here: these refusals must come before the first collective."""
    from vectisdb_b200.distributed import sharded_group_by
    node, arrays = _dense_case(3)
    with pytest.raises(ValueError, match="value type of AVG input"):
        sharded_group_by(node, lambda p: _group(p, arrays, False), {"x": T.FLOAT64})
    with pytest.raises(ValueError, match="GROUP BY node"):
        sharded_group_by(make_scan(["x"]), lambda p: [], TYPES)
    with pytest.raises(ValueError, match="wrong number of columns"):
        sharded_group_by(node, lambda p: _group(p, arrays, False)[:-1], TYPES)
