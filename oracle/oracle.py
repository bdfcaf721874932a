"""Test infrastructure (oracle side): the CPU restatement of the docking path.

Voxelization, rotation and top-t come from md_oracle.c (plain C, the
reference's float semantics); the FFTs, the conj(R^) product and the embedding
are numpy:
  * precision="fp64": complex128 FFTs (numpy pocketfft) -- the FP64 oracle;
  * precision="fp32": complex64 FFTs (scipy.fft) -- an FP32 stand-in.
The FFT is unnormalised with FFTW's signs (forward -1, inverse +1) as in
src/fft_process.cpp:349-396; the product is conj(R^) * L^ (:333-346); the
embedding puts the ng1^3 grids at offset ng1/2 (:306-330).

Only tests, the smoke check and the benchmark's CPU baseline leg use this.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libmd_oracle.so"

_FP = C.POINTER(C.c_float)
_IP = C.POINTER(C.c_int)
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise RuntimeError(f"{LIB} missing; run `make -C oracle restatement`")
        _lib = C.CDLL(str(LIB))
    return _lib


def _f(a):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_FP)


def rotation_matrix(theta):
    th = np.ascontiguousarray(theta, np.float32)
    m = np.zeros(9, np.float32)
    lib().oracle_rotation_matrix(_f(th), _f(m))
    return m


def rotate(xyz_centred, m9):
    xyz = np.ascontiguousarray(xyz_centred, np.float32).reshape(-1)
    m = np.ascontiguousarray(m9, np.float32)
    out = np.zeros_like(xyz)
    lib().oracle_rotate(len(xyz) // 3, _f(xyz), _f(m), _f(out))
    return out.reshape(-1, 3)


def ligand_grids(xyz_rot, radius, charge, ng1, grid_width, grid_coord, delta=1.0):
    xr = np.ascontiguousarray(xyz_rot, np.float32).reshape(-1)
    rad = np.ascontiguousarray(radius, np.float32)
    q = np.ascontiguousarray(charge, np.float32)
    gc = np.ascontiguousarray(grid_coord, np.float32)
    gr = np.zeros(ng1 ** 3, np.float32)
    gi = np.zeros(ng1 ** 3, np.float32)
    lib().oracle_ligand_grids(C.c_int(len(rad)), _f(xr), _f(rad), _f(q), C.c_int(ng1), C.c_float(grid_width),
                              _f(gc), C.c_float(delta), _f(gr), _f(gi))
    return gr.reshape((ng1,) * 3), gi.reshape((ng1,) * 3)


def score_sort(raw, t):
    r = np.ascontiguousarray(raw, np.float32)
    nf = r.shape[0]
    s = np.zeros(t, np.float32)
    idx = np.zeros(3 * t, np.int32)
    lib().oracle_score_sort(_f(r.reshape(-1)), C.c_int(nf), C.c_int(t), _f(s), idx.ctypes.data_as(_IP))
    return s, idx.reshape(-1, 3)


def embed(grid_r, grid_i, nf1, dtype=np.complex128):
    ng = grid_r.shape[0]
    off = (nf1 - ng) // 2
    z = np.zeros((nf1,) * 3, dtype)
    z[off:off + ng, off:off + ng, off:off + ng] = grid_r.astype(np.float64) + 1j * grid_i.astype(np.float64)
    return z


def _fftn(a, precision):
    if precision == "fp64":
        return np.fft.fftn(a.astype(np.complex128))
    import scipy.fft as sf
    return sf.fftn(a.astype(np.complex64), workers=-1)


def _ifftn_unnormalised(a, precision):
    n = a.size
    if precision == "fp64":
        return np.fft.ifftn(a.astype(np.complex128)) * n
    import scipy.fft as sf
    return sf.ifftn(a.astype(np.complex64), workers=-1, norm="forward")


def receptor_spectrum(grid_r, grid_i, nf1, precision="fp64"):
    return _fftn(embed(grid_r, grid_i, nf1), precision)


def raw_scores(rhat, lig_r, lig_i, precision="fp64"):
    """Unnormalised real part of IFFT(conj(R^) * FFT(L)) (float32 array)."""
    nf1 = rhat.shape[0]
    L = _fftn(embed(lig_r, lig_i, nf1), precision)
    P = np.conj(rhat) * L
    out = _ifftn_unnormalised(P, precision)
    return np.ascontiguousarray(out.real.astype(np.float32))


def raw_scores_f64(rhat, lig_r, lig_i):
    """Same in float64 without the final rounding (for tolerance studies)."""
    nf1 = rhat.shape[0]
    L = np.fft.fftn(embed(lig_r, lig_i, nf1))
    return (np.fft.ifftn(np.conj(rhat.astype(np.complex128)) * L) * L.size).real


def dock_rotation(rhat, xyz_centred, radius, charge, theta_or_m, ng1, grid_width, grid_coord, t, delta=1.0,
                  precision="fp64"):
    m = np.asarray(theta_or_m, np.float32)
    if m.size == 3:
        m = rotation_matrix(m)
    xr = rotate(xyz_centred, m)
    gr, gi = ligand_grids(xr, radius, charge, ng1, grid_width, grid_coord, delta)
    raw = raw_scores(rhat, gr, gi, precision)
    return score_sort(raw, t)
