"""torch.autograd.Function over md_adjoint_lse, for tests only.

LSEDock(rec_r, rec_u, charge, alpha) = T * log(sum_r exp(s_r / T)) with s_r
the top-1 score of rotation r when the receptor grids are (rec_r,
alpha * rec_u) and the ligand carries the given per-atom charges; the
forward runs the device docking path (md_receptor_fft, md_ligand_data,
md_dock with t = 1) and the backward the device adjoint.  Tensors live on the
CPU (the C ABI takes host buffers); the docking itself runs on the GPU.
"""
import numpy as np
import torch


class LSEDock(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rec_r, rec_u, charge, alpha, fp, job, rotmats, temperature):
        xyz, rad, _ = job.ligand_atoms()
        a = float(alpha)
        rr = rec_r.detach().numpy().astype(np.float32)
        ri = (np.float32(a) * rec_u.detach().numpy()).astype(np.float32)
        fp.receptor_fft(rr, ri)
        fp.ligand_data_transfer_gpu(xyz, rad, charge.detach().numpy().astype(np.float32), job.lig_core)
        top1 = fp.cuda_fft(rotmats, t=1)
        res = fp.adjoint_lse(rotmats, top1, temperature, a)
        ctx.save_for_backward(rec_u)
        ctx.res = res
        ctx.alpha = a
        return torch.tensor(res["loss"], dtype=torch.float64)

    @staticmethod
    def backward(ctx, gout):
        (rec_u,) = ctx.saved_tensors
        res = ctx.res
        g = float(gout)
        d_rec_r = torch.from_numpy(res["d_rec_r"]) * g
        d_rec_u = torch.from_numpy(res["d_rec_i"]) * (g * ctx.alpha)
        d_charge = torch.from_numpy(res["d_charge"]) * g
        d_alpha = torch.tensor(res["d_alpha"] * g, dtype=torch.float64)
        return d_rec_r, d_rec_u, d_charge, d_alpha, None, None, None, None
