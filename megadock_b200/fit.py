"""Fitting the electrostatic weight and per-residue charge scales with the
device adjoint, on decoys the docking path itself generates.

For every planted complex (megadock_b200.synth.plant_complex) the native
pose (the set rotation and grid translation that restore the planted ligand)
is the positive; the per-rotation top-1 poses of a docking run whose ligand
C-alphas lie more than `neg_rmsd` A (RMSD) from the native are the negatives.
The ranking loss of a pair is the softmax cross-entropy of the positive
against its negatives at temperature T:

    L_p = -s_pos + T * log(exp(s_pos / T) + sum_d exp(s_d / T))

Parameters: alpha, the electrostatic weight (the receptor's imaginary grid is
alpha * sum_k c_k U_k, U_k the field of the receptor atoms of residue type k
at unit weight, support fixed), and c_k, one charge scale per residue type,
applied to the receptor's and the ligand's charges alike.  Gradients:

    dL/dalpha = sum_x dL/dRi(x) * sum_k c_k U_k(x)
    dL/dc_k   = alpha * sum_x dL/dRi(x) U_k(x) + sum_{a in k} q0_a dL/dq_a

with dL/dRi and dL/dq from md_adjoint_poses (weights dL/ds per pose).
"""
from __future__ import annotations

import numpy as np

from ._native import POSE_DTYPE, rotation_matrices
from .fft_process import FFTProcess, Job
from .synth import AA_FREQ

RESIDUES = sorted(AA_FREQ)


def residue_codes(pdb_path) -> np.ndarray:
    """Residue-type index (RESIDUES order; len(RESIDUES) for anything else)
    of every heavy atom, in the order MEGADOCK reads them
    (src/pdb_entry.cpp:40-49: ATOM/HETATM records, hydrogens skipped by
    columns 77-78)."""
    index = {r: i for i, r in enumerate(RESIDUES)}
    out = []
    for line in open(pdb_path):
        if line.startswith(("ATOM  ", "HETATM")) and line[76:78] != " H":
            out.append(index.get(line[17:20].strip(), len(RESIDUES)))
    return np.asarray(out, np.int32)


def pose_rmsd(poses, mats, lig_file_ca, lig_center, rec_center, native_ca, nfft, grid_width) -> np.ndarray:
    """Ligand C-alpha RMSD to native_ca of each pose (rotation index into
    mats, translation i/j/k read as signed for >= nfft/2), the ligand placed
    as in megadock_b200.synth.decoy_ca: x_i = M y_i + b with y_i = ca_i -
    lig_center, b = rec_center - t * gw.  The sum over atoms of
    |M y_i + b - n_i|^2 is formed from 3x3 moments of y and the native n, so
    the cost per pose does not grow with the chain length."""
    t = np.stack([poses["i"], poses["j"], poses["k"]], -1).astype(np.int64)
    t = np.where(t >= nfft // 2, t - nfft, t)
    M = np.asarray(mats, np.float64)[poses["rot"]].reshape(-1, 3, 3)
    b = np.asarray(rec_center, np.float64) - t * grid_width
    y = np.asarray(lig_file_ca, np.float64) - lig_center
    x = np.asarray(native_ca, np.float64)
    n = len(y)
    Syy = y.T @ y                      # sum y y^T
    Syx = y.T @ x                      # sum y x^T
    sy, sx, sxx = y.sum(0), x.sum(0), float((x * x).sum())
    my = M @ sy                        # M sum y, per pose
    ssq = (np.einsum("pij,jk,pik->p", M, Syy, M) + n * (b * b).sum(-1) + sxx + 2 * (b * my).sum(-1)
           - 2 * np.einsum("pij,ji->p", M, Syx) - 2 * b @ sx)
    return np.sqrt(np.maximum(ssq, 0.0) / n)


class FitPair:
    """One planted complex on the device: its docking context, the receptor's
    per-residue-type field grids and the native pose."""

    def __init__(self, planted, nfft, rotation_set, device=0, batch=None, tune=False):
        self.pc = planted
        self.job = Job(["-R", planted.rec_pdb, "-L", planted.lig_pdb, "-F", str(nfft), "-r", str(rotation_set)])
        job = self.job
        self.N = job.nf1
        self.fp = FFTProcess(device)
        self.fp.alloc_array(job.nf1, job.grid_width, job.grid_coord())
        self.rec_r, _ = job.receptor_grids()
        self.rec_codes = residue_codes(planted.rec_pdb)
        self.lig_codes = residue_codes(planted.lig_pdb)
        self.K = len(RESIDUES) + 1
        self.U = job.receptor_elec_groups(self.rec_codes, self.K).reshape(self.K, -1)
        self.xyz, self.rad, self.q0 = job.ligand_atoms()
        self.mats = rotation_matrices(job.rotation_angles())
        self.rec_c, self.lig_c = [np.asarray(c, np.float64) for c in job.centers()]
        shift = np.asarray(planted.shift)
        if np.any(np.abs(shift) >= self.N // 2):
            raise ValueError("native translation outside the FFT box")
        self.pos = np.zeros(1, POSE_DTYPE)
        self.pos["rot"] = planted.rot_index
        self.pos["i"], self.pos["j"], self.pos["k"] = shift % self.N
        self.batch = batch
        if batch:
            self.fp.set_batch(batch)
        if tune:
            # launch shape of this FFT size (cached per size by the autotuner)
            import torch

            from .tune import autotune
            self.set_params(1.0, np.ones(self.K))
            d_rot = torch.from_numpy(self.mats).to(f"cuda:{device}")
            d_out = torch.zeros(len(self.mats) * 5, dtype=torch.int32, device=f"cuda:{device}")
            self.batch, _ = autotune(self.fp, d_rot.data_ptr(), d_out.data_ptr(), 1, sample=min(768, len(self.mats)))

    def set_params(self, alpha, scale):
        scale = np.asarray(scale, np.float64)
        ri = (alpha * (scale @ self.U)).astype(np.float32).reshape(self.rec_r.shape)
        self.fp.receptor_fft(self.rec_r, ri)
        q = (scale[self.lig_codes] * self.q0).astype(np.float32)
        self.fp.ligand_data_transfer_gpu(self.xyz, self.rad, q, self.job.lig_core)

    def rmsd(self, poses) -> np.ndarray:
        """Ligand C-alpha RMSD of each pose to the native."""
        return pose_rmsd(poses, self.mats, self.pc.lig_file_ca, self.lig_c, self.rec_c, self.pc.native_ca, self.N,
                         self.job.grid_width)

    def native_rmsd_check(self) -> float:
        """RMSD of the native pose to the planted ligand (0 up to rounding)."""
        return float(self.rmsd(self.pos)[0])

    def forward(self):
        """Per-rotation top-1 poses and the positive's score."""
        top1 = self.fp.cuda_fft(self.mats, t=1).copy()
        s_pos = float(self.fp.pose_scores(self.mats[self.pos["rot"]], self.pos)[0])
        return top1, s_pos

    def loss_grad(self, alpha, scale, temperature, neg_rmsd=10.0):
        """(loss, dL/dalpha, dL/dc, stats) of this pair at the current parameters
        (set_params must have been called with the same alpha and scale)."""
        top1, s_pos = self.forward()
        neg = top1[self.rmsd(top1) > neg_rmsd]
        s = np.concatenate([[s_pos], neg["score"].astype(np.float64)])
        m = s.max()
        e = np.exp((s - m) / temperature)
        z = e.sum()
        loss = -s_pos + m + temperature * np.log(z)
        p = e / z
        w = p.copy()
        w[0] -= 1.0
        live = np.concatenate([[True], neg["score"] > 0])    # clamped scores carry no gradient
        w[~live] = 0.0
        wf = w.astype(np.float32)
        keep = np.flatnonzero(wf != 0)
        poses = np.concatenate([self.pos, neg])[keep]
        g = self.fp.adjoint_poses(self.mats[poses["rot"]], poses, wf[keep])
        # the rotation work buffers (GBs at large launch groups) are freed
        # between evaluations so that every pair's context fits on the device
        self.fp.release_work()
        dri = g["d_rec_i"].reshape(-1).astype(np.float64)
        scale = np.asarray(scale, np.float64)
        d_alpha = float(dri @ (scale @ self.U))
        d_scale = alpha * (self.U @ dri)
        d_scale += np.bincount(self.lig_codes, weights=self.q0 * g["d_charge"], minlength=self.K)
        rank = int((s[1:] > s_pos).sum())
        return loss, d_alpha, d_scale, {"rank": rank, "n_neg": len(neg), "n_adj": len(keep), "s_pos": s_pos,
                                        "entries": np.concatenate([self.pos, neg]), "dl_ds": w,
                                        "d_rec_i": g["d_rec_i"], "d_charge": g["d_charge"]}


class Fitter:
    """Gradient descent (Adam) on alpha and the per-residue charge scales
    over a set of planted complexes."""

    def __init__(self, pairs, alpha=1.0, temperature=10.0, lr=0.05, neg_rmsd=10.0):
        self.pairs = pairs
        self.alpha = float(alpha)
        self.scale = np.ones(pairs[0].K)
        self.T = temperature
        self.lr = lr
        self.neg_rmsd = neg_rmsd
        self._m = np.zeros(1 + len(self.scale))
        self._v = np.zeros(1 + len(self.scale))
        self._n = 0

    def evaluate(self):
        """Mean loss and gradient over the pairs at the current parameters."""
        tot, ga, gs, stats = 0.0, 0.0, np.zeros_like(self.scale), []
        for p in self.pairs:
            p.set_params(self.alpha, self.scale)
            l, a, s, st = p.loss_grad(self.alpha, self.scale, self.T, self.neg_rmsd)
            tot += l
            ga += a
            gs += s
            stats.append(st)
        n = len(self.pairs)
        return tot / n, ga / n, gs / n, stats

    def step(self):
        loss, ga, gs, stats = self.evaluate()
        g = np.concatenate([[ga], gs])
        self._n += 1
        self._m = 0.9 * self._m + 0.1 * g
        self._v = 0.999 * self._v + 0.001 * g * g
        mh = self._m / (1 - 0.9 ** self._n)
        vh = self._v / (1 - 0.999 ** self._n)
        d = self.lr * mh / (np.sqrt(vh) + 1e-12)
        self.alpha -= d[0]
        self.scale = self.scale - d[1:]
        return loss, stats
