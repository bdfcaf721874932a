"""cuFFT comparator for the docking scores.

The same per-rotation scores as the fused pipeline, computed the way the
reference's GPU path does (fft_process.cpp:502-656): the ligand grids of a
rotation embedded at offset ng1/2 in an N^3 complex64 grid, a C2C forward
transform, the pointwise conj(R^) L^ product, a C2C inverse transform, and the
real part divided by N^3 (score = Re / nf3, fft_process.cpp:399-458).  The
transforms are the CUDA FFT library's, reached through torch.fft on a CUDA
device.

This module is a checker: the tests compare the fused kernels' poses and
receptor spectrum with it and the benchmark times it beside the fused path.
Nothing in the docking path calls it.  The ligand grids come from the
library's own voxelizer (md_ligand_voxels), which is bit-exact with the
reference's, so the comparison isolates the transform, product and top-t.
"""
from __future__ import annotations

import numpy as np


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("the cuFFT comparator needs a CUDA device")
    return torch


def embed(grid_r, grid_i, nf1: int, device="cuda"):
    """(B, ng, ng, ng) or (ng, ng, ng) real/imag grids -> complex64 N^3 grids
    with the ng^3 block at offset (N - ng) / 2 on each axis."""
    torch = _torch()
    gr = torch.as_tensor(np.asarray(grid_r, np.float32), device=device)
    gi = torch.as_tensor(np.asarray(grid_i, np.float32), device=device)
    single = gr.dim() == 3
    if single:
        gr, gi = gr[None], gi[None]
    b, ng = gr.shape[0], gr.shape[1]
    off = (nf1 - ng) // 2
    z = torch.zeros((b, nf1, nf1, nf1), dtype=torch.complex64, device=device)
    z[:, off:off + ng, off:off + ng, off:off + ng] = torch.complex(gr, gi)
    return z[0] if single else z


def receptor_spectrum(grid_r, grid_i, nf1: int, device="cuda"):
    """R^ = unnormalised forward C2C transform of the embedded receptor grids."""
    torch = _torch()
    return torch.fft.fftn(embed(grid_r, grid_i, nf1, device), dim=(-3, -2, -1))


def scores(rhat, lig):
    """Score grids Re(IFFT(conj(R^) FFT(L))) / N^3 for a batch of embedded
    ligand grids lig (B, N, N, N) complex64 -> (B, N, N, N) float32."""
    torch = _torch()
    lhat = torch.fft.fftn(lig, dim=(-3, -2, -1))
    # torch's inverse with the default normalisation divides by N^3, which is
    # the reference's division of the unnormalised result by nf3
    return torch.fft.ifftn(torch.conj(rhat) * lhat, dim=(-3, -2, -1)).real


def top_t(score_grids, t: int):
    """Top t scores per rotation and their (i, j, k) cells: (B, t) float32 and
    (B, t, 3) int64 on the host (ties broken by torch.topk, not the reference's
    index order; callers compare with a tolerance)."""
    torch = _torch()
    b, n = score_grids.shape[0], score_grids.shape[-1]
    v, i = torch.topk(score_grids.reshape(b, -1), t, dim=1)
    i = i.cpu().numpy()
    ijk = np.stack([i // (n * n), (i // n) % n, i % n], axis=-1)
    return v.cpu().numpy(), ijk


def cell_scores(score_grids, cells):
    """Scores at given cells: cells (B, t, 3) -> (B, t) float32 on the host."""
    torch = _torch()
    c = torch.as_tensor(np.asarray(cells, np.int64), device=score_grids.device)
    b = torch.arange(score_grids.shape[0], device=score_grids.device)[:, None].expand(c.shape[0], c.shape[1])
    return score_grids[b, c[..., 0], c[..., 1], c[..., 2]].cpu().numpy()
