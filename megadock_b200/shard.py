"""Rotation sharding of one docking job over the ranks of a process group.

MEGADOCK spreads the rotations of a job over the GPUs of one process
(src/docking.cpp:239-259, each GPU keeping its own copy of the receptor
spectrum, src/fft_process.cpp:263-272) and merges the per-rotation records
on the host.  Here every rank (one process per GPU, torch.distributed) docks
a contiguous block of the rotation set on its own device; the only exchange
is the gather of the per-rotation records (t x 20 bytes per rotation) on
rank 0, which merges them and writes the .out exactly as a one-GPU run does.
"""
from __future__ import annotations

import numpy as np

from ._native import POSE_DTYPE, rotation_matrices
from .fft_process import FFTProcess, Job


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous block [r0, r1) of n rotations for `rank` of `world`
    (sizes differ by at most one)."""
    base, extra = divmod(n, world)
    r0 = rank * base + min(rank, extra)
    return r0, r0 + base + (1 if rank < extra else 0)


def gather_poses(local: np.ndarray, group=None):
    """Concatenate every rank's records in rank order on rank 0 (None on the
    other ranks)."""
    import torch.distributed as dist
    rank = dist.get_rank(group)
    out = [None] * dist.get_world_size(group) if rank == 0 else None
    dist.gather_object(np.ascontiguousarray(local).view(POSE_DTYPE).tobytes(), out, dst=0, group=group)
    if rank != 0:
        return None
    return np.concatenate([np.frombuffer(b, POSE_DTYPE) for b in out])


def gather_records(local, nrot: int, t: int, group=None):
    """Every rank's block of pose records (an int32 tensor of n_local x t x 5
    words: score bits, rotation, i, j, k, the md_pose layout, for the block
    shard_range(nrot, rank, world)) concatenated in rotation order, on every
    rank: one all-gather of equal-size padded blocks over the group's backend
    (NCCL on the GPUs, gloo on the CPU).  This is the exchange step of a
    sharded job, the gather of MEGADOCK's per-rotation records."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    words = t * 5
    block = -(-nrot // world) * words
    buf = torch.zeros(block, dtype=torch.int32, device=local.device)
    buf[:local.numel()] = local.reshape(-1)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out = []
    for r in range(world):
        r0, r1 = shard_range(nrot, r, world)
        out.append(parts[r][:(r1 - r0) * words])
    return torch.cat(out)


def max_over_ranks(value: float, device=None, group=None) -> float:
    """The largest value over the ranks of the group (timings: a sharded job
    ends when its slowest rank does)."""
    import torch
    import torch.distributed as dist
    v = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(v, op=dist.ReduceOp.MAX, group=group)
    return float(v.item())


def torchrun_command(script: str, argv: list[str], nproc: int, port: int) -> list[str]:
    """Command that runs `script argv` as nproc ranks on this node, one per
    GPU (torch.distributed.run, rendezvous on 127.0.0.1)."""
    import sys
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={nproc}",
            "--master-addr", "127.0.0.1", f"--master-port={port}", script, *argv]


def _gpu_dock(job: Job, mats: np.ndarray, r0: int, r1: int, device: int, batch: int | None):
    fp = FFTProcess(device)
    fp.alloc_array(job.nf1, job.grid_width, job.grid_coord())
    rr, ri = job.receptor_grids()
    fp.receptor_fft(rr, ri)
    xyz, rad, q = job.ligand_atoms()
    fp.ligand_data_transfer_gpu(xyz, rad, q, job.lig_core)
    if batch:
        fp.set_batch(batch)
    poses = fp.cuda_fft(mats[r0:r1], t=job.t, first_rot=r0).copy()
    fp.fft_memory_free()
    return poses


def dock_sharded(args, device: int = 0, batch: int | None = 64, dock=None, group=None) -> Job:
    """Dock the job of MEGADOCK command line `args` with its rotations split
    over the ranks of `group`; rank 0 writes the .out.  `dock(job, mats, r0,
    r1)` replaces the device docking of a block (it must return the block's
    n x t records)."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    job = Job(args)
    mats = rotation_matrices(job.rotation_angles())
    r0, r1 = shard_range(job.n_rot, rank, world)
    local = (dock or (lambda j, m, a, b: _gpu_dock(j, m, a, b, device, batch)))(job, mats, r0, r1)
    if len(local) != (r1 - r0) * job.t:
        raise ValueError("a block must return t records per rotation")
    merged = gather_poses(local, group)
    if rank == 0:
        job.write_out(merged)
    return job
