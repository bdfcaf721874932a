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


def _stub_records(nrot, t, r0, r1):
    """int32 pose words (score bits, rot, i, j, k) of rotations [r0, r1)."""
    import torch
    rec = torch.zeros((r1 - r0, t, 5), dtype=torch.int32)
    for r in range(r0, r1):
        for j in range(t):
            score = torch.tensor([float((r * 7919 + 13 * j) % 997) + 0.25 * j], dtype=torch.float32)
            rec[r - r0, j, 0] = score.view(torch.int32)[0]
            rec[r - r0, j, 1:] = torch.tensor([r, (r * 3 + j) % 64, (r * 5) % 64, (r * 7 + j) % 64])
    return rec.reshape(-1)


def _gather_worker(rank, world, port, nrot, t, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from megadock_b200.shard import gather_records, max_over_ranks, shard_range
        r0, r1 = shard_range(nrot, rank, world)
        got = gather_records(_stub_records(nrot, t, r0, r1), nrot, t)
        ok = torch.equal(got, _stub_records(nrot, t, 0, nrot))
        slowest = max_over_ranks(10.0 + rank)
        q.put((rank, ok, slowest))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nrot", [(2, 361), (3, 100), (4, 7)])
def test_gather_records_in_rotation_order(world, nrot):
    """The benchmark's sharded step: each rank holds the records of its block
    (uneven blocks included); after the all-gather every rank holds the whole
    job's records in rotation order, and the step time is the slowest rank's."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    mp.spawn(_gather_worker, args=(world, _free_port(), nrot, 3, q), nprocs=world, join=True)
    res = sorted(q.get() for _ in range(world))
    assert [r[0] for r in res] == list(range(world))
    assert all(r[1] for r in res)
    assert all(r[2] == 10.0 + world - 1 for r in res)


def test_torchrun_command():
    import sys

    from megadock_b200.shard import torchrun_command
    cmd = torchrun_command("/x/bench.py", ["--gpus", "4", "--steps", "2"], 4, 29500)
    assert cmd[:3] == [sys.executable, "-m", "torch.distributed.run"]
    assert "--nproc-per-node=4" in cmd and "--master-addr" in cmd and "127.0.0.1" in cmd
    assert cmd[-5:] == ["/x/bench.py", "--gpus", "4", "--steps", "2"]
