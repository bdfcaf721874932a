"""Batched docking of many receptor-ligand pairs of uneven grid sizes.

MEGADOCK docks one pair per process and farms pairs out with MPI
(src/mpidp.cpp:281-551).  Here every pair gets a device context (its receptor
spectrum and ligand stay resident) and one captured CUDA graph runs the
rotations of all pairs back to back on a runner context's shared work
buffers (md_dock_pairs).

Rotations per launch and the inverse plane kernel's radix plan are chosen per
FFT size by the autotuner (megadock_b200.tune).

Grid choice: each pair uses the smallest N = 2 * ng with ng a 2^a 3^b 5^c
number (even, so the zero-padded half is aligned) that covers the complex by
MEGADOCK's sizing rule (Control::autogridr/l, src/control.cpp:287-379:
receptor bounding-box edge + 16 A, ligand maximum extent + 6 A, at 1.2 A per
cell) and has a built kernel set.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _native as N
from ._native import MdError, POSE_DTYPE
from .fft_process import FFTProcess, Job, _check


def _smooth235(n: int) -> bool:
    for p in (2, 3, 5):
        while n % p == 0:
            n //= p
    return n == 1


def _pdb_xyz(path):
    xyz = []
    for line in open(path):
        if line.startswith(("ATOM  ", "HETATM")) and line[76:78] != " H":
            xyz.append((float(line[30:38]), float(line[38:46]), float(line[46:54])))
    return np.asarray(xyz, np.float64)


def required_ng(rec_pdb, lig_pdb, grid_width=1.2, margin_rec=8.0, margin_lig=3.0) -> int:
    r = _pdb_xyz(rec_pdb)
    l = _pdb_xyz(lig_pdb)
    rec = float((r.max(0) - r.min(0)).max()) + 2 * margin_rec
    d = np.sqrt(((l[:, None, :] - l[None, :, :]) ** 2).sum(-1)).max() if len(l) > 1 else 0.0
    lig = float(d) + 2 * margin_lig
    return 1 + int(max(rec, lig) / grid_width)


def choose_fft_size(rec_pdb, lig_pdb, grid_width=1.2) -> int:
    ng = required_ng(rec_pdb, lig_pdb, grid_width)
    while True:
        if ng % 2 == 0 and _smooth235(ng) and N.lib().md_fft_size_supported(2 * ng):
            return 2 * ng
        ng += 1
        if ng > 512:
            raise MdError(N.MD_ERR_SIZE, "no built FFT size covers this complex")


class PairBatch:
    """All pairs of one batched run (contexts, device rotation sets, outputs)."""

    def __init__(self, pair_files, rotation_set=3600, t=1, device=0, extra_args=(), autotune=True, stream=None):
        import torch

        self.t = t
        self.device = device
        self.jobs, self.ctxs = [], []
        for rp, lp in pair_files:
            nf = choose_fft_size(rp, lp)
            job = None
            while job is None:
                try:
                    job = Job(["-R", rp, "-L", lp, "-F", str(nf), "-r", str(rotation_set), "-t", str(t),
                               *extra_args])
                except MdError as e:
                    if e.code != N.MD_ERR_SIZE:
                        raise
                    nf += 4                      # float rounding at the edge of a size: next size up
                    while not N.lib().md_fft_size_supported(nf) or not _smooth235(nf // 2):
                        nf += 4
            fp = FFTProcess(device)
            fp.alloc_array(job.nf1, job.grid_width, job.grid_coord())
            job.receptor_to(fp)
            xyz, rad, q = job.ligand_atoms()
            fp.ligand_data_transfer_gpu(xyz, rad, q, job.lig_core)
            self.jobs.append(job)
            self.ctxs.append(fp)
        from ._native import rotation_matrices
        mats = rotation_matrices(self.jobs[0].rotation_angles())
        self.n_rot = len(mats)
        self.d_rot = torch.from_numpy(mats).to(f"cuda:{device}")
        self.d_out = [torch.zeros(self.n_rot * t * 5, dtype=torch.int32, device=f"cuda:{device}")
                      for _ in self.ctxs]
        self.batch_by_n, self.plan_by_n, self.tile_by_n = {}, {}, {}
        if autotune:
            from .tune import autotune
            for fp in self.ctxs:
                if fp.num_fft not in self.batch_by_n:
                    self.batch_by_n[fp.num_fft], self.plan_by_n[fp.num_fft] = autotune(
                        fp, self.d_rot.data_ptr(), self.d_out[0].data_ptr(), t, sample=min(768, self.n_rot))
                    self.tile_by_n[fp.num_fft] = fp.tile
        for fp in self.ctxs:
            fp.set_batch(self.batch_by_n.get(fp.num_fft, 16))
            fp.set_plan(self.plan_by_n.get(fp.num_fft, 0))
            fp.set_tile(self.tile_by_n.get(fp.num_fft, 32))
        self.runner = FFTProcess(device, stream=stream)

    def run(self, stream=None):
        """Enqueue every pair's rotations as one graph on the runner's stream."""
        n = len(self.ctxs)
        ctxs = (C.c_void_p * n)(*[fp._h.value for fp in self.ctxs])
        rots = (C.c_void_p * n)(*([self.d_rot.data_ptr()] * n))
        nrot = (C.c_int * n)(*([self.n_rot] * n))
        outs = (C.c_void_p * n)(*[o.data_ptr() for o in self.d_out])
        _check(N.lib().md_dock_pairs(self.runner._h, ctxs, n, rots, nrot, self.t, outs), self.runner._h)

    def poses(self):
        import torch
        torch.cuda.synchronize(self.device)
        return [o.cpu().numpy().view(POSE_DTYPE) for o in self.d_out]

    def sizes(self):
        return [fp.num_fft for fp in self.ctxs]


def uneven_workload(npairs=64, rotation_set=3600, t=1, seed_base=2000, outdir=None, device=0, stream=None):
    """The uneven-pairs workload: pairs with chain lengths log-uniform in
    60-800 residues (megadock_b200.synth.uneven_pairs)."""
    import tempfile

    from . import synth
    outdir = outdir or tempfile.mkdtemp(prefix="md_pairs_")
    files = [synth.write_pair(outdir, nr, nl, seed, stem=f"p{seed}")
             for nr, nl, seed in synth.uneven_pairs(npairs, seed_base)]
    return PairBatch(files, rotation_set=rotation_set, t=t, device=device, stream=stream)
