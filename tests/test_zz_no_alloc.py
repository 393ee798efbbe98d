"""vgpu_group_by_count_sum_noalloc -- the group-by entry point for callers that cannot allocate device
memory (a host callback, a graph-driven loop, memory reserved by another allocator) -- against the
general entry point, vgpu_execute_plan, and against the plan oracle, on the same data. Two calls in a
row with different key ranges also show that the shared scratch array starts clean on every call;
rows whose keys lie outside the declared range are skipped; work queued on a side stream is ordered
on that stream. Counts are bit-exact; the DOUBLE sums are accumulated with atomics, so their order (and
last bits) vary from run to run, and they are compared within 1e-12 relative. Collected last on
purpose."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-12


def _reference(keys, values):
    from vectisdb_b200 import GpuEngine, make_aggregate, make_column, make_group_by, make_scan
    from vectisdb_b200.engine import GpuAggregateKind as A, GpuValueType as T
    plan = make_group_by(["k"], [make_aggregate(A.COUNT_STAR, "", T.INT64), make_aggregate(A.SUM, "v", T.FLOAT64)],
                         make_scan(["k", "v"]))
    r = GpuEngine.instance().execute_plan(plan, [make_column("k", T.INT32, keys), make_column("v", T.FLOAT64, values)])
    assert r.success, r.error_message
    k, c, s = [col.data for col in r.columns]
    order = np.argsort(k)
    return k[order], c[order], s[order]


def _oracle(keys, values):
    from oracle.plan_oracle import evaluate
    from vectisdb_b200 import make_aggregate, make_column, make_group_by, make_scan
    from vectisdb_b200.engine import GpuAggregateKind as A, GpuValueType as T
    plan = make_group_by(["k"], [make_aggregate(A.COUNT_STAR, "", T.INT64), make_aggregate(A.SUM, "v", T.FLOAT64)],
                         make_scan(["k", "v"]))
    k, c, s = [np.asarray(col.data) for col in evaluate(plan, [make_column("k", T.INT32, keys),
                                                               make_column("v", T.FLOAT64, values)])]
    order = np.argsort(k)
    return k[order], c[order], s[order]


def _noalloc(keys, values, key_min, domain, stream=None):
    import torch
    from vectisdb_b200 import abi
    dev = torch.device("cuda:0")
    dk = torch.from_numpy(keys).to(dev)
    dv = torch.from_numpy(values).to(dev)
    ok_ = torch.empty(domain, dtype=torch.int32, device=dev)
    oc = torch.empty(domain, dtype=torch.int64, device=dev)
    osum = torch.empty(domain, dtype=torch.float64, device=dev)
    og = torch.empty(1, dtype=torch.int64, device=dev)
    if stream is None:
        stream = torch.cuda.current_stream()
    else:  # inputs and outputs were made on the current stream: the side stream waits for them
        stream.wait_stream(torch.cuda.current_stream())
    status = abi.lib().vgpu_group_by_count_sum_noalloc(
        C.c_void_p(dk.data_ptr()), C.c_void_p(dv.data_ptr()), len(keys), key_min, domain,
        C.c_void_p(ok_.data_ptr()), C.c_void_p(oc.data_ptr()), C.c_void_p(osum.data_ptr()),
        C.c_void_p(og.data_ptr()), C.c_void_p(stream.cuda_stream))
    assert status == abi.OK, abi.last_error()
    stream.synchronize()
    g = int(og.item())
    return ok_[:g].cpu().numpy(), oc[:g].cpu().numpy(), osum[:g].cpu().numpy()


def _data(seed, n, lo, hi):
    rng = np.random.default_rng(seed)
    return rng.integers(lo, hi, n).astype(np.int32), rng.random(n)


def test_noalloc_group_by_matches_execute_plan_twice_in_a_row():
    for seed, n, lo, hi in [(1, 1_000_003, -500, 1500), (2, 200_000, 7, 300)]:
        keys, values = _data(seed, n, lo, hi)
        got = _noalloc(keys, values, lo, hi - lo)
        exp = _reference(keys, values)
        assert np.array_equal(got[0], exp[0])
        assert np.array_equal(got[1], exp[1])
        assert np.all(np.abs(got[2] - exp[2]) <= REL * np.abs(exp[2]))


def _check(got, exp):
    assert np.array_equal(got[0], exp[0])
    assert np.array_equal(got[1], exp[1])
    assert np.all(np.abs(got[2] - exp[2]) <= REL * np.abs(exp[2]))


def test_noalloc_skips_keys_outside_its_range_on_a_side_stream():
    """Keys reach 300 below and above [key_min, key_min + domain): only the rows inside count, as in the
    oracle's and vgpu_execute_plan's group-by over those rows; two calls in a row on a side stream."""
    import torch
    side = torch.cuda.Stream()
    for seed, n, lo, hi in [(3, 300_001, -200, 900), (4, 150_000, 40, 41 + 65535 - 600)]:
        keys, values = _data(seed, n, lo - 300, hi + 300)
        inside = (keys >= lo) & (keys < hi)
        assert inside.sum() < n  # some rows do lie outside
        got = _noalloc(keys, values, lo, hi - lo, stream=side)
        _check(got, _oracle(keys[inside], values[inside]))
        _check(got, _reference(keys[inside], values[inside]))


def test_noalloc_matches_the_oracle():
    keys, values = _data(5, 250_000, -1000, 3000)
    _check(_noalloc(keys, values, -1000, 4000), _oracle(keys, values))


def test_noalloc_rejects_a_domain_beyond_its_scratch():
    from vectisdb_b200 import abi
    import torch
    torch.cuda.init()
    status = abi.lib().vgpu_group_by_count_sum_noalloc(None, None, 0, 0, 1 << 17, None, None, None, None, None)
    assert status == abi.ERR_INVALID_ARGUMENT
    assert "65536" in abi.last_error()
