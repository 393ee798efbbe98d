"""The collective step of the device-merged sharded GROUP BY (distributed.exchange_rows), with two gloo
ranks on the CPU: each rank routes rows of packed-key words to their owners the way vgpu_shard_route
orders them (owner = MurmurHash3's 64-bit finalizer of the key, mod world; rows grouped by owner), the
rows cross in one all-to-all, and every rank must receive exactly the rows it owns, from both ranks,
sender by sender -- including a rank that sends nothing and a round where nobody sends anything."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rows(rank, n, words=5):
    rng = np.random.default_rng(100 + rank)
    rows = rng.integers(0, 1 << 40, size=(n, words), dtype=np.int64)
    rows[:, 1] = rank  # sender tag
    return rows


def _routed(rows, world):
    """Rows grouped by owner (stable within an owner) and the rows per owner."""
    from vectisdb_b200.distributed import _owner
    owner = _owner(rows[:, 0], world)
    order = np.argsort(owner, kind="stable")
    return rows[order], np.bincount(owner, minlength=world).tolist()


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    from vectisdb_b200.distributed import exchange_rows
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        for case, n in (("both", 3000 + 517 * rank), ("one_empty", 2000 if rank == 0 else 0), ("none", 0)):
            send, splits = _routed(_rows(rank, n), world)
            recv = exchange_rows(torch.from_numpy(send), splits)
            out[(case, rank)] = (send, splits, recv.numpy())
        try:
            exchange_rows(torch.zeros((3, 2), dtype=torch.int64), [1, 1])  # counts that miss a row
            out[("bad", rank)] = "sent"
        except ValueError as e:
            out[("bad", rank)] = str(e)
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module")
def results():
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    return dict(out)


@pytest.mark.parametrize("case", ["both", "one_empty", "none"])
def test_every_rank_receives_exactly_the_rows_it_owns(results, case):
    from vectisdb_b200.distributed import _owner
    for r in range(2):
        _, _, recv = results[(case, r)]
        assert np.all(_owner(recv[:, 0], 2) == r)
        # sender by sender: rank 0's rows for r, then rank 1's, each in the order they were sent
        want = []
        for s in range(2):
            send, splits, _ = results[(case, s)]
            start = sum(splits[:r])
            want.append(send[start:start + splits[r]])
        assert np.array_equal(recv, np.concatenate(want))


def test_row_counts_that_do_not_cover_the_rows_are_refused(results):
    assert "one row count per rank" in results[("bad", 0)]
    assert "one row count per rank" in results[("bad", 1)]
