"""Sharded group-by merge (vectisdb_b200.distributed): two gloo ranks on the CPU each aggregate half of
the rows, the partial groups are merged with all-reduces, and the result must equal the aggregation of
all rows -- exactly for counts, MIN/MAX and 128-bit integer sums (values near 2^62 make the sums leave
64 bits), within 1e-12 relative for FP64 sums. One rank with no rows contributes identities."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _data(seed):
    rng = np.random.default_rng(seed)
    n = 20000
    k = rng.integers(-50, 200, n)
    k[rng.random(n) < 0.2] = 7  # one heavy key
    x = rng.standard_normal(n)
    v = rng.integers((1 << 62) - 1000, 1 << 62, n, dtype=np.int64)
    v[rng.random(n) < 0.3] *= -1
    w = rng.integers(-(1 << 40), 1 << 40, n, dtype=np.int64)
    return k, x, v, w


def _partial(k, x, v, w):
    """What a rank's engine run returns: its groups with SUM(x), SUM(v) as HUGEINT, COUNT(*), MIN/MAX(w)."""
    sys.path.insert(0, ROOT)
    from vectisdb_b200.distributed import HUGEINT
    keys = np.unique(k)
    pos = np.searchsorted(keys, k)
    sx = np.zeros(len(keys))
    np.add.at(sx, pos, x)
    cnt = np.bincount(pos, minlength=len(keys)).astype(np.int64)
    mn = np.full(len(keys), np.iinfo(np.int64).max)
    np.minimum.at(mn, pos, w)
    mx = np.full(len(keys), np.iinfo(np.int64).min)
    np.maximum.at(mx, pos, w)
    sv = np.zeros(len(keys), HUGEINT)
    for i, key in enumerate(keys.tolist()):
        total = int(v[k == key].astype(object).sum())
        sv[i]["lower"] = total & ((1 << 64) - 1)
        u = (total >> 64) & ((1 << 64) - 1)
        sv[i]["upper"] = u - (1 << 64) if u >= (1 << 63) else u
    return keys, [("sum_f64", sx), ("sum_i128", sv), ("count", cnt), ("min", mn), ("max", mx)]


def _rank(rank, world, port, seed, empty_rank, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    from vectisdb_b200.distributed import merge_dense_groupby
    k, x, v, w = _data(seed)
    lo, hi = (0, len(k) // 2) if rank == 0 else (len(k) // 2, len(k))
    if rank == empty_rank:
        lo = hi = 0
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        keys, aggs = _partial(k[lo:hi], x[lo:hi], v[lo:hi], w[lo:hi])
        mk, magg = merge_dense_groupby(keys, aggs, -50, 199)
        out[rank] = (mk, magg)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("empty_rank", [-1, 1])
def test_merge_of_two_ranks_equals_the_whole(empty_rank):
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, 5, empty_rank, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    k, x, v, w = _data(5)
    if empty_rank == 1:  # rank 1 contributed nothing: the whole is rank 0's half
        half = len(k) // 2
        k, x, v, w = k[:half], x[:half], v[:half], w[:half]
    ek, eaggs = _partial(k, x, v, w)
    for rank in (0, 1):
        mk, magg = out[rank]
        assert np.array_equal(mk, ek)
        sx, sv, cnt, mn, mx = magg
        assert np.all(np.abs(sx - eaggs[0][1]) <= 1e-12 * np.maximum(np.abs(eaggs[0][1]), 1e-300) + 1e-12)
        assert np.array_equal(sv["lower"], eaggs[1][1]["lower"]) and np.array_equal(sv["upper"], eaggs[1][1]["upper"])
        assert np.array_equal(cnt, eaggs[2][1]) and np.array_equal(mn, eaggs[3][1]) and np.array_equal(mx, eaggs[4][1])


def test_sparse_domains_and_unknown_kinds_are_refused_before_any_collective():
    """No process group exists here: each refusal must come before the first collective."""
    sys.path.insert(0, ROOT)
    from vectisdb_b200.distributed import merge_dense_groupby
    with pytest.raises(ValueError, match="not dense"):
        merge_dense_groupby(np.array([0]), [("count", np.array([1]))], 0, 1 << 24)
    with pytest.raises(ValueError, match="does not merge"):
        merge_dense_groupby(np.array([0]), [("avg", np.array([1.0]))], 0, 10)
    with pytest.raises(ValueError, match="one value per key"):
        merge_dense_groupby(np.array([0, 1]), [("count", np.array([1]))], 0, 10)
    with pytest.raises(ValueError, match="outside"):
        merge_dense_groupby(np.array([11]), [("count", np.array([1]))], 0, 10)


def _hc_data(seed):
    rng = np.random.default_rng(seed)
    n = 60000
    k = rng.integers(0, 1 << 40, 30000)[rng.integers(0, 30000, n)]  # ~25k distinct sparse keys
    k[rng.random(n) < 0.1] = 12345  # a heavy key
    x = rng.standard_normal(n)
    v = rng.integers((1 << 62) - 1000, 1 << 62, n, dtype=np.int64)
    v[rng.random(n) < 0.4] *= -1
    w = rng.integers(-(1 << 40), 1 << 40, n, dtype=np.int64)
    return k, x, v, w


def _rank_repart(rank, world, port, seed, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    from vectisdb_b200.distributed import repartition_merge_groupby
    k, x, v, w = _hc_data(seed)
    lo, hi = (0, len(k) // 3) if rank == 0 else (len(k) // 3, len(k))  # uneven halves
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        keys, aggs = _partial(k[lo:hi], x[lo:hi], v[lo:hi], w[lo:hi])
        out[rank] = repartition_merge_groupby(keys, aggs)
    finally:
        dist.destroy_process_group()


def test_repartition_merge_of_high_cardinality_groups():
    """Sparse 40-bit keys: each rank ends with the groups its hash owns -- disjoint shares that together
    equal the aggregation of all rows."""
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_repart, args=(r, 2, port, 9, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(240)
        assert p.exitcode == 0
    ek, eaggs = _partial(*_hc_data(9))
    k0, a0 = out[0]
    k1, a1 = out[1]
    assert len(np.intersect1d(k0, k1)) == 0 and len(k0) > 0 and len(k1) > 0
    keys = np.concatenate([k0, k1])
    order = np.argsort(keys)
    assert np.array_equal(keys[order], ek)
    sx = np.concatenate([a0[0], a1[0]])[order]
    sv = np.concatenate([a0[1], a1[1]])[order]
    rest = [np.concatenate([a0[i], a1[i]])[order] for i in (2, 3, 4)]
    assert np.all(np.abs(sx - eaggs[0][1]) <= 1e-12 * np.maximum(np.abs(eaggs[0][1]), 1e-300) + 1e-12)
    assert np.array_equal(sv["lower"], eaggs[1][1]["lower"]) and np.array_equal(sv["upper"], eaggs[1][1]["upper"])
    for got, (_, exp) in zip(rest, eaggs[2:]):
        assert np.array_equal(got, exp)


def test_i128_to_f64_rounds_like_python_ints():
    """The AVG finish's 128-bit -> double conversion is the nearest double, ties to even, like Python's
    int -> float: values at the int64 edges, ties above 2^53 and values far outside 64 bits."""
    sys.path.insert(0, ROOT)
    from vectisdb_b200.distributed import HUGEINT, _i128_to_f64
    rng = np.random.default_rng(11)
    vals = [0, 1, -1, (1 << 53) + 1, (1 << 53) + 3, -(1 << 53) - 1, (1 << 63) - 1, -(1 << 63), 1 << 63, -(1 << 63) - 1,
            (1 << 64) + 2048, (1 << 100) + (1 << 47), -(1 << 127), (1 << 127) - 1]
    vals += [int(x) for x in rng.integers(-(1 << 62), 1 << 62, 200)]
    vals += [int(x) * (1 << 40) + int(y) for x, y in zip(rng.integers(-(1 << 60), 1 << 60, 200),
                                                        rng.integers(0, 1 << 40, 200))]
    arr = np.zeros(len(vals), HUGEINT)
    for i, v in enumerate(vals):
        arr[i]["lower"] = v & ((1 << 64) - 1)
        u = (v >> 64) & ((1 << 64) - 1)
        arr[i]["upper"] = u - (1 << 64) if u >= 1 << 63 else u
    got = _i128_to_f64(arr)
    assert [float(v) for v in vals] == got.tolist()


def _rank_reagg(rank, world, port, seed, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    from oracle.plan_oracle import evaluate
    from vectisdb_b200.distributed import repartition_merge_groupby
    k, x, v, w = _hc_data(seed)
    lo, hi = (0, len(k) // 3) if rank == 0 else (len(k) // 3, len(k))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        keys, aggs = _partial(k[lo:hi], x[lo:hi], v[lo:hi], w[lo:hi])
        pos = np.searchsorted(keys, k[lo:hi])  # MIN/MAX of the DOUBLE column x merge as floats
        xmn = np.full(len(keys), np.inf)
        np.minimum.at(xmn, pos, x[lo:hi])
        xmx = np.full(len(keys), -np.inf)
        np.maximum.at(xmx, pos, x[lo:hi])
        aggs += [("min_f64", xmn), ("max_f64", xmx)]
        plain = repartition_merge_groupby(keys, aggs)
        calls = []

        def run(plan, columns):  # the plan oracle standing in for the engine's GROUP BY
            calls.append([a.kind for a in plan.aggregates])
            return evaluate(plan, columns)

        out[rank] = (plain, repartition_merge_groupby(keys, aggs, reaggregate=run), calls)
    finally:
        dist.destroy_process_group()


def test_repartition_merge_through_a_group_by_executor():
    """The received partials re-aggregated by a GROUP BY executor (the engine's, in a deployment) give
    the numpy merge's result: counts, MIN/MAX and 128-bit sums exactly (the sums travel as four 32-bit
    chunk columns), FP64 sums within 1e-12 relative."""
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_reagg, args=(r, 2, port, 13, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(240)
        assert p.exitcode == 0
    for rank in (0, 1):
        (pk, pa), (rk, ra), calls = out[rank]
        # SUM f64, 4 chunk SUMs, COUNT, MIN, MAX, float MIN, float MAX
        assert len(calls) == 1 and len(calls[0]) == 1 + 4 + 1 + 1 + 1 + 2
        assert np.array_equal(pk, rk) and len(pk) > 0
        assert np.all(np.abs(ra[0] - pa[0]) <= 1e-12 * np.abs(pa[0]) + 1e-12)
        assert np.array_equal(ra[1]["lower"], pa[1]["lower"]) and np.array_equal(ra[1]["upper"], pa[1]["upper"])
        for got, want in zip(ra[2:], pa[2:]):
            assert got.dtype == want.dtype and np.array_equal(got, want)
        assert pa[5].dtype == np.float64 and np.any(pa[5] != np.round(pa[5])) and np.any(pa[5] < 0)
    k, x, _, _ = _hc_data(13)  # the float MIN/MAX equal those over all rows
    keys = np.concatenate([out[0][0][0], out[1][0][0]])
    order = np.argsort(keys)
    ek = np.unique(k)
    assert np.array_equal(keys[order], ek)
    pos = np.searchsorted(ek, k)
    emn = np.full(len(ek), np.inf)
    np.minimum.at(emn, pos, x)
    emx = np.full(len(ek), -np.inf)
    np.maximum.at(emx, pos, x)
    assert np.array_equal(np.concatenate([out[0][0][1][5], out[1][0][1][5]])[order], emn)
    assert np.array_equal(np.concatenate([out[0][0][1][6], out[1][0][1][6]])[order], emx)
