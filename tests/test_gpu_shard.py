"""Rotation sharding with the device path: two gloo ranks on the one GPU
here (independent processes; nothing waits across them on the device) dock
halves of the rotation set, and rank 0's .out equals the one-process
megadock-b200 output of the same command line."""
import os
import socket
import subprocess

import pytest

pytestmark = pytest.mark.gpu


def _worker(rank, world, port, args):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from megadock_b200.shard import dock_sharded
        dock_sharded(args, device=0)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_match_single_run(built, gpu, pairs, tmp_path):
    import torch.multiprocessing as mp

    from megadock_b200 import _native
    rp, lp = pairs["c0"]
    common = ["-R", rp, "-L", lp, "-F", "96", "-r", "3600", "-t", "2", "-N", "500"]
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    sharded, single = tmp_path / "sharded.out", tmp_path / "single.out"
    mp.spawn(_worker, args=(2, port, common + ["-o", str(sharded)]), nprocs=2, join=True)
    r = subprocess.run([str(_native.CLI_PATH), *common, "-o", str(single)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    assert sharded.read_text() == single.read_text()
