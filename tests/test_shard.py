"""Rotation sharding on the CPU: the block split covers every rotation once,
and a two-rank gloo group that docks halves of the rotation set (a stub
stands in for the device) writes, on rank 0, the same .out as one process
writing all records (the gather and merge path of megadock_b200.shard)."""
import os
import socket

import numpy as np
import pytest


def test_shard_range_partition():
    from megadock_b200.shard import shard_range
    for n in (1, 7, 3600, 54000):
        for world in (1, 2, 3, 8):
            blocks = [shard_range(n, r, world) for r in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == n
            assert all(blocks[r][1] == blocks[r + 1][0] for r in range(world - 1))
            sizes = [b - a for a, b in blocks]
            assert max(sizes) - min(sizes) <= 1


def _stub_dock(job, mats, r0, r1):
    from megadock_b200 import POSE_DTYPE
    out = np.zeros((r1 - r0) * job.t, POSE_DTYPE)
    for r in range(r0, r1):
        for j in range(job.t):
            e = out[(r - r0) * job.t + j]
            e["score"] = float((r * 7919 + 13 * j) % 997) + 0.25 * j
            e["rot"], e["i"], e["j"], e["k"] = r, (r * 3 + j) % job.nf1, (r * 5) % job.nf1, (r * 7 + j) % job.nf1
            out[(r - r0) * job.t + j] = e
    return out


def _worker(rank, world, port, args):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from megadock_b200.shard import dock_sharded
        dock_sharded(args, dock=_stub_dock)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_out_equals_single_process(built, pairs, tmp_path, world):
    import torch.multiprocessing as mp

    from megadock_b200 import Job, rotation_matrices
    rp, lp = pairs["small"]
    sharded = tmp_path / f"sharded{world}.out"
    single = tmp_path / "single.out"
    common = ["-R", rp, "-L", lp, "-F", "64", "-r", "360", "-t", "2", "-N", "100"]
    mp.spawn(_worker, args=(world, _free_port(), common + ["-o", str(sharded)]), nprocs=world, join=True)
    job = Job(common + ["-o", str(single)])
    job.write_out(_stub_dock(job, rotation_matrices(job.rotation_angles()), 0, job.n_rot))
    assert sharded.read_text() == single.read_text()
    assert len(sharded.read_text().splitlines()) == 4 + 100
