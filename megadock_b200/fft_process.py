"""Python mirror of MEGADOCK's docking-path interface over the C ABI.

``FFTProcess`` keeps the method names and argument meaning of the reference's
class (src/fft_process.h:168-195) so callers and tests read like MEGADOCK's
own driver (src/docking.cpp:194-346): alloc_array, receptor_fft,
ligand_data_transfer_gpu, cuda_fft, sort_index, top_score, top_index,
fft_memory_free.  Errors raise ``MdError`` instead of calling exit().

``Job`` mirrors ``Control`` (src/control.cpp): a MEGADOCK command line parsed,
sized and run end to end, writing the same .out file.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from ._native import MdError, POSE_DTYPE


def _check(rc, ctx=None, what=""):
    if rc:
        msg = N.lib().md_last_error(ctx).decode() if ctx else what
        raise MdError(rc, msg or what)


class FFTProcess:
    """Device context for one receptor-ligand pair on one GPU."""

    def __init__(self, device: int = 0, stream: int | None = None):
        h = C.c_void_p()
        _check(N.lib().md_ctx_create(device, C.byref(h)), None, "md_ctx_create")
        self._h = h
        self.num_fft = 0
        self._top = None
        self.plan, self.tile, self.lanes = 0, 32, 2
        if stream is not None:
            _check(N.lib().md_set_stream(self._h, C.c_void_p(stream)), self._h)

    # -- FFTProcess::alloc_array(num_fft) + Docking::rec_init grid coordinates
    def alloc_array(self, num_fft: int, grid_width: float, grid_coord: np.ndarray):
        gc = np.ascontiguousarray(grid_coord, dtype=np.float32)
        _check(N.lib().md_set_grid(self._h, int(num_fft), float(grid_width), N.fptr(gc)), self._h)
        self.num_fft = int(num_fft)

    # -- FFTProcess::receptor_fft(grid_r, grid_i)
    def receptor_fft(self, grid_r: np.ndarray, grid_i: np.ndarray):
        r = np.ascontiguousarray(grid_r, dtype=np.float32)
        i = np.ascontiguousarray(grid_i, dtype=np.float32)
        _check(N.lib().md_receptor_fft(self._h, N.fptr(r), N.fptr(i)), self._h)

    def receptor_build(self, xyz_centred, radius, charge, ace, rec_core=-45.0, ace_ratio=1.0, elec_ratio=1.0,
                       make_receptor=True, return_grids=False):
        """Receptor grids built on the device (md_receptor_build); with
        make_receptor they become this context's receptor, like receptor_fft."""
        xyz = np.ascontiguousarray(xyz_centred, dtype=np.float32).reshape(-1)
        rad = np.ascontiguousarray(radius, dtype=np.float32)
        q = np.ascontiguousarray(charge, dtype=np.float32)
        a = np.ascontiguousarray(ace, dtype=np.float32)
        ng = self.num_fft // 2
        gr = np.zeros(ng ** 3, np.float32) if return_grids else None
        gi = np.zeros(ng ** 3, np.float32) if return_grids else None
        _check(N.lib().md_receptor_build(self._h, len(rad), N.fptr(xyz), N.fptr(rad), N.fptr(q), N.fptr(a),
                                         float(rec_core), float(ace_ratio), float(elec_ratio), int(make_receptor),
                                         N.fptr(gr) if gr is not None else None,
                                         N.fptr(gi) if gi is not None else None), self._h)
        if return_grids:
            return gr.reshape((ng,) * 3), gi.reshape((ng,) * 3)

    def receptor_spectrum(self) -> np.ndarray:
        n3 = self.num_fft ** 3
        re = np.zeros(n3, np.float32)
        im = np.zeros(n3, np.float32)
        _check(N.lib().md_receptor_spectrum(self._h, N.fptr(re), N.fptr(im)), self._h)
        return (re + 1j * im.astype(np.complex64)).reshape((self.num_fft,) * 3)

    # -- FFTProcess::ligand_data_transfer_gpu(grid_coord)
    def ligand_data_transfer_gpu(self, xyz_centred, radius, charge, lig_core: float = 1.0):
        xyz = np.ascontiguousarray(xyz_centred, dtype=np.float32).reshape(-1)
        rad = np.ascontiguousarray(radius, dtype=np.float32)
        q = np.ascontiguousarray(charge, dtype=np.float32)
        _check(N.lib().md_ligand_data(self._h, len(rad), N.fptr(xyz), N.fptr(rad), N.fptr(q), float(lig_core)),
               self._h)
        self._na = len(rad)

    def set_batch(self, rotations_per_launch: int):
        _check(N.lib().md_set_batch(self._h, int(rotations_per_launch)), self._h)

    def release_work(self):
        """Free the rotation work buffers (allocated again by the next call)."""
        _check(N.lib().md_release_work(self._h), self._h)

    def set_tile(self, lines: int):
        """kz lines per CTA of the x-line kernel (8, 16 or 32)."""
        _check(N.lib().md_set_tile(self._h, int(lines)), self._h)
        self.tile = int(lines)

    def set_lanes(self, lanes: int):
        """Launch groups of the batched form in flight at once (1 or 2)."""
        _check(N.lib().md_set_lanes(self._h, int(lanes)), self._h)
        self.lanes = int(lanes)

    def set_plan(self, plan: int):
        """Radix plan variant of the inverse plane kernel (0, 1 or 2)."""
        _check(N.lib().md_set_plan(self._h, int(plan)), self._h)
        self.plan = int(plan)

    # -- FFTProcess::cuda_fft over a rotation range
    def cuda_fft(self, rotmats: np.ndarray, t: int = 1, first_rot: int = 0) -> np.ndarray:
        m = np.ascontiguousarray(rotmats, dtype=np.float32).reshape(-1, 9)
        out = np.zeros(len(m) * t, POSE_DTYPE)
        _check(N.lib().md_dock(self._h, N.fptr(m), int(first_rot), len(m), int(t), N.vptr(out)), self._h)
        self._top = out
        return out

    def dock_device(self, d_rotmat: int, first_rot: int, n_rot: int, t: int, d_out: int):
        _check(N.lib().md_dock_device(self._h, C.c_void_p(d_rotmat), first_rot, n_rot, t, C.c_void_p(d_out)),
               self._h)

    def dock_profile(self, d_rotmat: int, first_rot: int, n_rot: int, t: int, d_out: int):
        """Per-stage device milliseconds (voxelize, plane_fwd, xline, plane_inv,
        merge) and the launch count."""
        ms = np.zeros(5, np.float32)
        nl = C.c_int()
        _check(N.lib().md_dock_profile(self._h, C.c_void_p(d_rotmat), first_rot, n_rot, t, C.c_void_p(d_out),
                                       N.fptr(ms), C.byref(nl)), self._h)
        return ms, nl.value

    def ligand_voxels(self, rotmat9: np.ndarray):
        m = np.ascontiguousarray(rotmat9, dtype=np.float32).reshape(9)
        ng = self.num_fft // 2
        r = np.zeros(ng ** 3, np.float32)
        i = np.zeros(ng ** 3, np.float32)
        _check(N.lib().md_ligand_voxels(self._h, N.fptr(m), N.fptr(r), N.fptr(i)), self._h)
        return r.reshape((ng,) * 3), i.reshape((ng,) * 3)

    def adjoint_lse(self, rotmats: np.ndarray, top1: np.ndarray, temperature: float = 10.0, alpha: float = 1.0,
                    lig_rot=()):
        """Gradient of T*log(sum_r exp(s_r/T)) over the top-1 scores s_r of
        md_dock (t = 1) poses.  Returns a dict: loss, d_rec_r, d_rec_i (ng^3),
        d_charge (na), d_alpha and, for the rotation indices in lig_rot,
        d_lig_r / d_lig_i (len(lig_rot), ng, ng, ng)."""
        m = np.ascontiguousarray(rotmats, dtype=np.float32).reshape(-1, 9)
        top1 = np.ascontiguousarray(top1).view(N.POSE_DTYPE).reshape(-1)
        if len(top1) != len(m):
            raise ValueError("one top-1 pose per rotation")
        ng = self.num_fft // 2
        ng3 = ng ** 3
        na = self._na
        sel = np.ascontiguousarray(lig_rot, dtype=np.int32).reshape(-1)
        if sel.size and (sel.min() < 0 or sel.max() >= len(m)):
            raise ValueError("lig_rot index out of range")
        loss = C.c_double()
        dalpha = C.c_double()
        drr = np.zeros(ng3, np.float32)
        dri = np.zeros(ng3, np.float32)
        dq = np.zeros(max(na, 1), np.float32)
        dlr = np.zeros(max(sel.size, 1) * ng3, np.float32)
        dli = np.zeros(max(sel.size, 1) * ng3, np.float32)
        _check(N.lib().md_adjoint_lse(self._h, N.fptr(m), len(m), N.vptr(top1), float(temperature), float(alpha),
                                      C.byref(loss), N.fptr(drr), N.fptr(dri), N.fptr(dq), C.byref(dalpha),
                                      sel.ctypes.data_as(C.POINTER(C.c_int)), int(sel.size), N.fptr(dlr),
                                      N.fptr(dli)), self._h)
        shape = (ng,) * 3
        return {"loss": loss.value, "d_rec_r": drr.reshape(shape), "d_rec_i": dri.reshape(shape),
                "d_charge": dq[:na], "d_alpha": dalpha.value,
                "d_lig_r": dlr[:sel.size * ng3].reshape((sel.size,) + shape),
                "d_lig_i": dli[:sel.size * ng3].reshape((sel.size,) + shape)}

    def adjoint_poses(self, rotmats: np.ndarray, poses: np.ndarray, dl_ds: np.ndarray, lig_pose=()):
        """Gradient for a loss with dL/d(score of pose p) = dl_ds[p]; pose p has
        rotation matrix rotmats[p] and translation poses[p] i/j/k.  Returns a
        dict: d_rec_r, d_rec_i (ng^3), d_charge (na), d_lig_r / d_lig_i for the
        poses listed in lig_pose."""
        m = np.ascontiguousarray(rotmats, dtype=np.float32).reshape(-1, 9)
        poses = np.ascontiguousarray(poses).view(N.POSE_DTYPE).reshape(-1)
        w = np.ascontiguousarray(dl_ds, dtype=np.float32).reshape(-1)
        if not (len(m) == len(poses) == len(w)):
            raise ValueError("one rotation matrix and one weight per pose")
        ng3 = (self.num_fft // 2) ** 3
        sel = np.ascontiguousarray(lig_pose, dtype=np.int32).reshape(-1)
        drr = np.zeros(ng3, np.float32)
        dri = np.zeros(ng3, np.float32)
        dq = np.zeros(max(self._na, 1), np.float32)
        dlr = np.zeros(max(sel.size, 1) * ng3, np.float32)
        dli = np.zeros(max(sel.size, 1) * ng3, np.float32)
        _check(N.lib().md_adjoint_poses(self._h, N.fptr(m), len(m), N.vptr(poses), N.fptr(w), N.fptr(drr),
                                        N.fptr(dri), N.fptr(dq), sel.ctypes.data_as(C.POINTER(C.c_int)),
                                        int(sel.size), N.fptr(dlr), N.fptr(dli)), self._h)
        shape = ((self.num_fft // 2),) * 3
        return {"d_rec_r": drr.reshape(shape), "d_rec_i": dri.reshape(shape), "d_charge": dq[:self._na],
                "d_lig_r": dlr[:sel.size * ng3].reshape((sel.size,) + shape),
                "d_lig_i": dli[:sel.size * ng3].reshape((sel.size,) + shape)}

    def pose_scores(self, rotmats: np.ndarray, poses: np.ndarray) -> np.ndarray:
        """Scores of given poses (rotation matrix per pose, translation i/j/k)."""
        m = np.ascontiguousarray(rotmats, dtype=np.float32).reshape(-1, 9)
        poses = np.ascontiguousarray(poses).view(N.POSE_DTYPE).reshape(-1)
        if len(m) != len(poses):
            raise ValueError("one rotation matrix per pose")
        out = np.zeros(len(m), np.float32)
        _check(N.lib().md_pose_scores(self._h, N.fptr(m), len(m), N.vptr(poses), N.fptr(out)), self._h)
        return out

    # -- FFTProcess::sort_index / top_score / top_index
    def sort_index(self, nout: int):
        self._top = N.sort_poses(self._top, nout)

    def top_score(self, j: int) -> float:
        return float(self._top[j]["score"])

    def top_index(self, j: int, k: int) -> int:
        return int(self._top[j][("rot", "i", "j", "k")[k]])

    # -- FFTProcess::fft_memory_free
    def fft_memory_free(self):
        if getattr(self, "_h", None):
            N.lib().md_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.fft_memory_free()
        except Exception:
            pass


class Job:
    """A MEGADOCK command line (Control::initialize / Control::execute)."""

    def __init__(self, args):
        argv = ["megadock-b200"] + [str(a) for a in args]
        arr = (C.c_char_p * len(argv))(*[a.encode() for a in argv])
        h = C.c_void_p()
        rc = N.lib().md_job_create(len(argv), arr, C.byref(h))
        self._h = h
        if rc:
            msg = N.lib().md_job_error(h).decode()
            self.close()
            raise MdError(rc, msg)
        dims = [C.c_int() for _ in range(7)]
        N.lib().md_job_dims(self._h, *[C.byref(d) for d in dims])
        self.ng1, self.nf1, self.na_rec, self.na_lig, self.n_rot, self.t, self.n_out = [d.value for d in dims]
        self.grid_width = N.lib().md_job_grid_width(self._h)
        self.lig_core = N.lib().md_job_lig_core(self._h)

    @property
    def log(self) -> str:
        return N.lib().md_job_log(self._h).decode()

    @property
    def out_file(self) -> str:
        return N.lib().md_job_out_file(self._h).decode()

    def grid_coord(self):
        a = np.zeros(self.ng1, np.float32)
        N.lib().md_job_grid_coord(self._h, N.fptr(a))
        return a

    def receptor_grids(self):
        n = self.ng1 ** 3
        r = np.zeros(n, np.float32)
        i = np.zeros(n, np.float32)
        N.lib().md_job_receptor_grids(self._h, N.fptr(r), N.fptr(i))
        return r.reshape((self.ng1,) * 3), i.reshape((self.ng1,) * 3)

    def receptor_elec_groups(self, group, ngroups: int) -> np.ndarray:
        """The receptor's electrostatic grid split by atom group (ngroups grids
        of ng1^3; atom l goes to group[l], negative = left out)."""
        g = np.ascontiguousarray(group, dtype=np.int32)
        if len(g) != self.na_rec:
            raise ValueError("one group per receptor atom")
        out = np.zeros((ngroups,) + (self.ng1,) * 3, np.float32)
        rc = N.lib().md_job_receptor_elec_groups(self._h, g.ctypes.data_as(C.POINTER(C.c_int)), int(ngroups),
                                                 N.fptr(out))
        if rc:
            raise MdError(rc, "md_job_receptor_elec_groups")
        return out

    def ligand_atoms(self):
        xyz = np.zeros(3 * self.na_lig, np.float32)
        rad = np.zeros(self.na_lig, np.float32)
        q = np.zeros(self.na_lig, np.float32)
        N.lib().md_job_ligand_atoms(self._h, N.fptr(xyz), N.fptr(rad), N.fptr(q))
        return xyz.reshape(-1, 3), rad, q

    def receptor_atoms(self):
        n = self.na_rec
        xyz, rad, q, ace = (np.zeros(3 * n, np.float32), np.zeros(n, np.float32), np.zeros(n, np.float32),
                            np.zeros(n, np.float32))
        N.lib().md_job_receptor_atoms(self._h, N.fptr(xyz), N.fptr(rad), N.fptr(q), N.fptr(ace))
        return xyz.reshape(-1, 3), rad, q, ace

    def centers(self):
        r = np.zeros(3, np.float32)
        l = np.zeros(3, np.float32)
        N.lib().md_job_centers(self._h, N.fptr(r), N.fptr(l))
        return r, l

    def rotation_angles(self):
        a = np.zeros(3 * self.n_rot, np.float32)
        N.lib().md_job_rotation_angles(self._h, N.fptr(a))
        return a.reshape(-1, 3)

    def run(self, fft: FFTProcess | None = None):
        rc = N.lib().md_job_run(self._h, fft._h if fft else None)
        if rc:
            raise MdError(rc, N.lib().md_job_error(self._h).decode())

    def receptor_to(self, fft: FFTProcess):
        """Build this job's receptor grids on fft's device and make them its
        receptor (fft must hold this job's grid: alloc_array(nf1, ...))."""
        rc = N.lib().md_job_receptor_to(self._h, fft._h)
        if rc:
            raise MdError(rc, N.lib().md_last_error(fft._h).decode())

    def write_out(self, poses, fft: FFTProcess | None = None):
        """Merge n_rot * t poses (rotation-major) and write the .out file."""
        p = np.ascontiguousarray(poses).view(POSE_DTYPE).reshape(-1)
        rc = N.lib().md_job_write_out(self._h, fft._h if fft else None, N.vptr(p), len(p))
        if rc:
            raise MdError(rc, N.lib().md_job_error(self._h).decode())

    def poses(self):
        out = np.zeros(self.n_rot * self.t, POSE_DTYPE)
        N.lib().md_job_poses(self._h, N.vptr(out))
        return out

    def top(self):
        out = np.zeros(self.n_out, POSE_DTYPE)
        N.lib().md_job_top(self._h, N.vptr(out))
        return out

    def close(self):
        if getattr(self, "_h", None):
            N.lib().md_job_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
