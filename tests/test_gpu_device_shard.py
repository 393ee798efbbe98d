"""The device-side exchange of a GROUP BY split by rows across GPUs (vgpu_shard_* and
distributed.device_sharded_group_by) against the oracle.

Each case runs as a child process (tests/_device_shard_worker.py) with its own one-rank nccl process
group, so no process group of this test process is touched. One GPU: the all-to-all of a single rank
is a copy, and the routing to several owners is checked by routing one rank's partial groups to four
virtual owners and merging each owner's rows alone (two ranks on one GPU would put NCCL kernels that
wait on each other on one device, which is not done here)."""
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(mode: str):
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0", MASTER_ADDR="127.0.0.1",
               MASTER_PORT=str(_free_port()), NCCL_NVLS_ENABLE="0")
    p = subprocess.run([sys.executable, str(ROOT / "tests" / "_device_shard_worker.py"), mode], env=env, cwd=ROOT,
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0 and "OK" in p.stdout, p.stdout[-2000:] + p.stderr[-4000:]


@pytest.mark.gpu
def test_device_merged_high_cardinality_group_by_matches_oracle():
    _run("c1")


@pytest.mark.gpu
def test_device_merged_dense_group_by_matches_oracle():
    _run("c0")


@pytest.mark.gpu
def test_routing_to_four_owners_partitions_the_groups():
    _run("route4")
