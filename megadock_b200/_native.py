"""ctypes binding of libmd_b200.so (include/md_b200.h).

The library is built in-tree by ``megadock_b200.build.build()``; loading fails
loudly when it is missing -- there is no pure-Python or CPU fallback for the
docking path.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libmd_b200.so"
CLI_PATH = PKG / "bin" / "megadock-b200"

MD_OK, MD_ERR_ARG, MD_ERR_CUDA, MD_ERR_STATE, MD_ERR_SIZE, MD_ERR_IO, MD_ERR_USAGE = range(7)


class MdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[md status {code}] {msg}")
        self.code = code


class Pose(C.Structure):
    """md_pose: {score, rot, i, j, k} (MEGADOCK SortScore, src/fft_process.h:40-43)."""
    _fields_ = [("score", C.c_float), ("rot", C.c_int), ("i", C.c_int), ("j", C.c_int), ("k", C.c_int)]


POSE_DTYPE = np.dtype([("score", "<f4"), ("rot", "<i4"), ("i", "<i4"), ("j", "<i4"), ("k", "<i4")])

_FP = C.POINTER(C.c_float)
_IP = C.POINTER(C.c_int)
_VP = C.c_void_p
_CP = C.c_char_p

_PROTOS = {
    "md_ctx_create": (C.c_int, [C.c_int, C.POINTER(_VP)]),
    "md_ctx_destroy": (None, [_VP]),
    "md_last_error": (_CP, [_VP]),
    "md_set_stream": (C.c_int, [_VP, _VP]),
    "md_fft_size_supported": (C.c_int, [C.c_int]),
    "md_set_grid": (C.c_int, [_VP, C.c_int, C.c_float, _FP]),
    "md_receptor_fft": (C.c_int, [_VP, _FP, _FP]),
    "md_receptor_spectrum": (C.c_int, [_VP, _FP, _FP]),
    "md_ligand_data": (C.c_int, [_VP, C.c_int, _FP, _FP, _FP, C.c_float]),
    "md_set_batch": (C.c_int, [_VP, C.c_int]),
    "md_release_work": (C.c_int, [_VP]),
    "md_set_lanes": (C.c_int, [_VP, C.c_int]),
    "md_set_plan": (C.c_int, [_VP, C.c_int]),
    "md_set_tile": (C.c_int, [_VP, C.c_int]),
    "md_dock": (C.c_int, [_VP, _FP, C.c_int, C.c_int, C.c_int, _VP]),
    "md_dock_device": (C.c_int, [_VP, _VP, C.c_int, C.c_int, C.c_int, _VP]),
    "md_dock_pairs": (C.c_int, [_VP, C.POINTER(_VP), C.c_int, C.POINTER(_VP), C.POINTER(C.c_int), C.c_int,
                                C.POINTER(_VP)]),
    "md_ligand_voxels": (C.c_int, [_VP, _FP, _FP, _FP]),
    "md_adjoint_poses": (C.c_int, [_VP, _FP, C.c_int, _VP, _FP, _FP, _FP, _FP, _IP, C.c_int, _FP, _FP]),
    "md_pose_scores": (C.c_int, [_VP, _FP, C.c_int, _VP, _FP]),
    "md_pose_terms": (C.c_int, [_VP, _FP, _FP, C.c_int, _IP, _FP]),
    "md_receptor_build": (C.c_int, [_VP, C.c_int, _FP, _FP, _FP, _FP, C.c_float, C.c_float, C.c_float, C.c_int,
                                    _FP, _FP]),
    "md_adjoint_lse": (C.c_int, [_VP, _FP, C.c_int, _VP, C.c_float, C.c_float, C.POINTER(C.c_double), _FP, _FP, _FP,
                                 C.POINTER(C.c_double), _IP, C.c_int, _FP, _FP]),
    "md_dock_profile": (C.c_int, [_VP, _VP, C.c_int, C.c_int, C.c_int, _VP, _FP, _IP]),
    "md_dock_noalloc": (C.c_int, [C.c_int, C.c_float, _VP, _VP, C.c_int, _VP, _VP, _VP, C.c_float, _VP, C.c_int,
                                  C.c_int, C.c_int, _VP, _VP]),
    "md_rotation_matrix": (C.c_int, [_FP, _FP]),
    "md_sort_poses": (C.c_int, [_VP, C.c_int, C.c_int]),
    "md_job_create": (C.c_int, [C.c_int, C.POINTER(_CP), C.POINTER(_VP)]),
    "md_job_error": (_CP, [_VP]),
    "md_job_log": (_CP, [_VP]),
    "md_job_destroy": (None, [_VP]),
    "md_job_run": (C.c_int, [_VP, _VP]),
    "md_job_receptor_to": (C.c_int, [_VP, _VP]),
    "md_job_write_out": (C.c_int, [_VP, _VP, _VP, C.c_int]),
    "md_job_dims": (C.c_int, [_VP, _IP, _IP, _IP, _IP, _IP, _IP, _IP]),
    "md_job_grid_width": (C.c_float, [_VP]),
    "md_job_out_file": (_CP, [_VP]),
    "md_job_grid_coord": (C.c_int, [_VP, _FP]),
    "md_job_receptor_grids": (C.c_int, [_VP, _FP, _FP]),
    "md_job_ligand_atoms": (C.c_int, [_VP, _FP, _FP, _FP]),
    "md_job_receptor_atoms": (C.c_int, [_VP, _FP, _FP, _FP, _FP]),
    "md_job_receptor_elec_groups": (C.c_int, [_VP, _IP, C.c_int, _FP]),
    "md_decoy_pdb": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.c_char_p]),
    "md_ligand_centres": (C.c_int, [C.c_char_p, C.c_int, C.c_char_p]),
    "md_table_mode": (C.c_int, [C.c_int, C.POINTER(C.c_char_p)]),
    "md_table_run": (C.c_int, [C.c_int, C.POINTER(C.c_char_p), _VP, _IP, _IP]),
    "md_table_expand": (C.c_int, [C.c_int, C.POINTER(C.c_char_p), C.c_int, C.c_int, C.c_char_p, C.c_int, _IP]),
    "md_job_centers": (C.c_int, [_VP, _FP, _FP]),
    "md_job_rotation_angles": (C.c_int, [_VP, _FP]),
    "md_job_lig_core": (C.c_float, [_VP]),
    "md_job_poses": (C.c_int, [_VP, _VP]),
    "md_job_top": (C.c_int, [_VP, _VP]),
}

EXPORTED = sorted(_PROTOS)

_lib = None


def lib():
    """Load libmd_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise MdError(MD_ERR_STATE, f"{LIB_PATH} is missing; run megadock_b200.build.build() first")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _PROTOS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_FP)


def vptr(a: np.ndarray):
    assert a.flags.c_contiguous
    return C.c_void_p(a.ctypes.data)


def rotation_matrix(theta) -> np.ndarray:
    th = np.ascontiguousarray(theta, dtype=np.float32).reshape(3)
    m = np.zeros(9, np.float32)
    rc = lib().md_rotation_matrix(fptr(th), fptr(m))
    if rc:
        raise MdError(rc, "md_rotation_matrix")
    return m


def rotation_matrices(angles) -> np.ndarray:
    a = np.ascontiguousarray(angles, dtype=np.float32).reshape(-1, 3)
    out = np.zeros((a.shape[0], 9), np.float32)
    for r in range(a.shape[0]):
        out[r] = rotation_matrix(a[r])
    return out


def sort_poses(poses: np.ndarray, nout: int) -> np.ndarray:
    p = np.ascontiguousarray(poses.copy()).astype(POSE_DTYPE)
    rc = lib().md_sort_poses(vptr(p), len(p), nout)
    if rc:
        raise MdError(rc, "md_sort_poses")
    return p[:nout]


def data_dir() -> str:
    return os.environ.get("MD_B200_DATA", str(PKG / "data"))
