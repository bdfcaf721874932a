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
