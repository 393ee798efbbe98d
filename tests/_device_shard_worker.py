"""One rank of a device-merged sharded GROUP BY (run by tests/test_gpu_device_shard.py as a child process with
RANK/WORLD_SIZE/MASTER_* set, one GPU, nccl). Checks the merged groups against the oracle on the whole
table and exits non-zero on any difference.

Rank r of w holds rows [r*n/w, (r+1)*n/w) of a seeded table. Modes:
  c1: the high-cardinality shape (composite key, DECIMAL SUM, AVG(DOUBLE), COUNT(*), MAX) through
      device_sharded_group_by;
  c0: the filter + group-by shape (1024 groups, SUM(DOUBLE), COUNT, MIN, MAX);
  route4: one rank routes its partial groups to 4 virtual owners (vgpu_shard_route with world 4), each
      owner's rows re-aggregated on their own; the owners' key sets are disjoint and together give the
      oracle's result.
"""
import datetime
import os
import sys

import numpy as np
import torch
import torch.distributed as dist

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from oracle import oracle as O  # noqa: E402
from vectisdb_b200 import abi  # noqa: E402
from vectisdb_b200 import workloads as W  # noqa: E402
from vectisdb_b200.distributed import _owner, device_sharded_group_by  # noqa: E402
from vectisdb_b200.engine import GpuValueType as T, make_device_column  # noqa: E402


def close(got, exp, rel=1e-12):
    got, exp = np.asarray(got, np.float64), np.asarray(exp, np.float64)
    return got.shape == exp.shape and bool(np.all(np.abs(got - exp) <= rel * np.maximum(np.abs(exp), 1e-300)))


def device_inputs(wl, lo, hi):
    keep, cols = [], []
    for c in wl.inputs:
        t = torch.from_numpy(np.ascontiguousarray(c.data[lo:hi])).cuda()
        keep.append(t)
        cols.append(make_device_column(c.name, c.type, t.data_ptr(), hi - lo))
    return keep, cols


def check_c1(out, exp):
    d = {n: t.cpu().numpy() for n, t in out}
    order = np.lexsort((d["b"], d["a"]))
    a, b = d["a"][order], d["b"][order]
    s = d["agg_0"][order]
    ok = np.array_equal(a, exp["a"]) and np.array_equal(b, exp["b"])
    ok = ok and np.array_equal(s[:, 0].view(np.uint64), exp["sum_lo"]) and np.array_equal(s[:, 1], exp["sum_hi"])
    ok = ok and close(d["agg_1"][order], exp["avg"])
    ok = ok and np.array_equal(d["agg_2"][order], exp["count"]) and np.array_equal(d["agg_3"][order], exp["max"])
    return ok


def gather_all(out):
    """Every rank's share on every rank (host arrays), for the whole-table comparison."""
    shares = [None] * dist.get_world_size()
    dist.all_gather_object(shares, [(n, t.cpu().numpy()) for n, t in out])
    merged = []
    for j, (name, _) in enumerate(shares[0]):
        merged.append((name, torch.from_numpy(np.concatenate([s[j][1] for s in shares]))))
    return merged


def main():
    mode = sys.argv[1]
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    torch.cuda.set_device(0)
    abi.lib().vgpu_set_device(0)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=60))
    n = 1 << 20
    lo, hi = rank * n // world, (rank + 1) * n // world
    ok = True
    if mode == "c1":
        wl = W.c1(n=n, seed=7)
        keep, cols = device_inputs(wl, lo, hi)
        out = device_sharded_group_by(wl.plan, cols, {"v": T.FLOAT64})
        exp = O.c1(*[c.data for c in wl.inputs], wl.params["ts_gt"])
        ok = check_c1(gather_all(out), exp)
    elif mode == "c0":
        wl = W.c0(n=n, seed=8)
        keep, cols = device_inputs(wl, lo, hi)
        out = gather_all(device_sharded_group_by(wl.plan, cols, {}))
        d = {nm: t.numpy() for nm, t in out}
        exp = O.c0(*[c.data for c in wl.inputs], wl.params["v_lt"], wl.params["w_mod"])
        order = np.argsort(d["col0"] if "col0" in d else d[out[0][0]], kind="stable")
        k = out[0][1].numpy()[order]
        ok = np.array_equal(k, exp["k"]) and close(d["agg_0"][order], exp["sum"])
        ok = ok and np.array_equal(d["agg_1"][order], exp["count"])
        ok = ok and np.array_equal(d["agg_2"][order], exp["min"]) and np.array_equal(d["agg_3"][order], exp["max"])
    elif mode == "route4":
        ok = route4(n)
    dist.barrier()
    dist.destroy_process_group()
    print("OK" if ok else "MISMATCH", flush=True)
    sys.exit(0 if ok else 1)


def route4(n):
    """One GPU routes its partial groups to 4 virtual owners (vgpu_shard_route with world 4); each owner's
    rows are merged alone (columns, engine GROUP BY, finish). The owners' shares are disjoint and
    together equal the oracle's result; every routed row sits in its owner's range."""
    from vectisdb_b200.distributed import _partial_plan
    from vectisdb_b200.engine import GpuEngine
    wl = W.c1(n=n, seed=9)
    keep, cols = device_inputs(wl, 0, n)
    plan, kinds, finish, count_at = _partial_plan(wl.plan, {"v": T.FLOAT64}, "route4")
    eng = GpuEngine.instance()
    held = []
    side = torch.cuda.Stream()  # every call below is ordered on this one stream
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        return route4_on(wl, cols, plan, kinds, finish, count_at, eng, held, side.cuda_stream)


def route4_on(wl, cols, plan, kinds, finish, count_at, eng, held, sp):
    from vectisdb_b200.distributed import _merge_exchanged, _raw_column, _route_partials
    from vectisdb_b200.engine import DeviceResult, ExecuteOptions

    def run(p, c):
        r = eng.execute_plan(p, c, ExecuteOptions(output_on_device=True, stream=sp))
        assert isinstance(r, DeviceResult), r.error_message
        held.append(r)
        return r

    local = run(plan, cols)
    raw = [_raw_column(local, i) for i in range(len(local.columns))]
    a = wl.inputs[0].data
    b = wl.inputs[1].data
    lo = [int(a.min()), int(b.min())]  # bounds every group's key (the groups are a subset of the rows)
    bits = [int(a.max() - lo[0]).bit_length(), int(b.max() - lo[1]).bit_length()]
    shifts = [bits[1], 0]
    send, counts = _route_partials(raw, 2, kinds, lo, shifts, 4, sp)
    rows = int(raw[0].row_count)
    if sum(counts) != rows:
        return False
    hsend = send.cpu().numpy()
    owner = _owner(hsend[:, 0], 4)
    starts = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    for r in range(4):
        if not np.all(owner[starts[r]:starts[r + 1]] == r):
            return False
    shares = []
    for r in range(4):
        part = send[starts[r]:starts[r + 1]].contiguous()
        shares.append(_merge_exchanged(part, kinds, finish, count_at, ["a", "b"], [T.INT32, T.INT32], shifts, bits,
                                       lo, run, sp))
    torch.cuda.synchronize()
    merged = [(shares[0][j][0], torch.cat([sh[j][1] for sh in shares]).cpu()) for j in range(len(shares[0]))]
    for r in held:
        r.free()
    pk = (merged[0][1].numpy().astype(np.int64) << 32) | merged[1][1].numpy().astype(np.int64)
    if np.unique(pk).shape[0] != pk.shape[0]:  # the owners' shares are disjoint
        return False
    return check_c1(merged, O.c1(*[c.data for c in wl.inputs], wl.params["ts_gt"]))


if __name__ == "__main__":
    main()
