"""Test infrastructure (oracle side): ctypes access to the reference itself.

Loads oracle/_ref/libref_harness.so -- MEGADOCK's own CPU sources compiled
unmodified against the project-written FFTW-API shim (oracle/Makefile) -- and
exposes its state for parity checks.  Only tests, the smoke check and the CPU
baseline leg of the benchmark use this module.

Each RefSession runs in its own process (the reference keeps global state and
never frees a session); use ``run_in_subprocess`` for isolation.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
HARNESS = HERE / "_ref" / "libref_harness.so"
REF_BIN = HERE / "_ref" / "megadock-ref"

_FP = C.POINTER(C.c_float)
_IP = C.POINTER(C.c_int)


def available() -> bool:
    return HARNESS.exists() and REF_BIN.exists()


def _f(a):
    return a.ctypes.data_as(_FP)


def _i(a):
    return a.ctypes.data_as(_IP)


class RefSession:
    def __init__(self, args, fft="fp32"):
        os.environ["MD_SHIM_FFT"] = fft
        self.L = C.CDLL(str(HARNESS))
        argv = ["megadock-ref"] + [str(a) for a in args]
        arr = (C.c_char_p * len(argv))(*[a.encode() for a in argv])
        rc = self.L.ref_open(len(argv), arr)
        if rc:
            raise RuntimeError("ref_open failed")
        v = [C.c_int() for _ in range(7)]
        gw = C.c_float()
        self.L.ref_info(C.byref(v[0]), C.byref(v[1]), C.byref(gw), C.byref(v[2]), C.byref(v[3]), C.byref(v[4]),
                        C.byref(v[5]))
        self.ng1, self.nf1, self.na_lig, self.na_rec, self.n_rot, self.t = [x.value for x in v[:6]]
        self.grid_width = gw.value
        self._rec_done = False

    def grid_coord(self):
        self.rec_init()
        a = np.zeros(self.ng1, np.float32)
        self.L.ref_grid_coord(_f(a))
        return a

    def centers(self):
        r = np.zeros(3, np.float32)
        l = np.zeros(3, np.float32)
        self.L.ref_receptor_center(_f(r))
        self.L.ref_ligand_center(_f(l))
        return r, l

    def atoms(self, which):
        n = self.na_lig if which else self.na_rec
        xyz, rad, q, ace = (np.zeros(3 * n, np.float32), np.zeros(n, np.float32), np.zeros(n, np.float32),
                            np.zeros(n, np.float32))
        self.L.ref_atoms(int(which), _f(xyz), _f(rad), _f(q), _f(ace))
        return xyz.reshape(-1, 3), rad, q, ace

    def rec_init(self):
        if not self._rec_done:
            self.L.ref_rec_init()
            self._rec_done = True

    def receptor_grids(self):
        self.rec_init()
        n = self.ng1 ** 3
        r = np.zeros(n, np.float32)
        i = np.zeros(n, np.float32)
        self.L.ref_receptor_grids(_f(r), _f(i))
        return r.reshape((self.ng1,) * 3), i.reshape((self.ng1,) * 3)

    def spectrum(self):
        self.rec_init()
        n = self.nf1 ** 3
        re = np.zeros(n, np.float32)
        im = np.zeros(n, np.float32)
        self.L.ref_spectrum(_f(re), _f(im))
        return (re.astype(np.complex64) + 1j * im.astype(np.complex64)).reshape((self.nf1,) * 3)

    def angles(self, ang):
        th = np.zeros(3, np.float32)
        self.L.ref_rotation_angles(int(ang), _f(th))
        return th

    def ligand_grids(self, ang):
        self.rec_init()
        n = self.ng1 ** 3
        xyz = np.zeros(3 * self.na_lig, np.float32)
        r = np.zeros(n, np.float32)
        i = np.zeros(n, np.float32)
        self.L.ref_ligand_grids(int(ang), _f(xyz), _f(r), _f(i))
        return xyz.reshape(-1, 3), r.reshape((self.ng1,) * 3), i.reshape((self.ng1,) * 3)

    def dock_rotation(self, ang):
        """(scores[t], index[t,4]) of the reference's CPU chain for one rotation."""
        self.rec_init()
        s = np.zeros(self.t, np.float32)
        idx = np.zeros(4 * self.t, np.int32)
        self.L.ref_dock_rotation(int(ang), _f(s), _i(idx))
        return s, idx.reshape(-1, 4)

    def score_grid(self):
        raw = np.zeros(self.nf1 ** 3, np.float32)
        self.L.ref_score_grid(_f(raw))
        return raw.reshape((self.nf1,) * 3)


def run_in_subprocess(fn, *args, **kw):
    """Run fn(*args) in a fresh spawned process (reference state is global)."""
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        return pool.apply(fn, args, kw)
