"""Generate the golden fixtures of the headline workload from the reference itself.

Test infrastructure: runs the reference's own CPU program and its C-ABI harness
(oracle/_ref, MEGADOCK's CPU sources compiled unmodified against the project's
FFTW-API shim, see oracle/Makefile) on the bench pair -- the 500/250-residue
synthetic receptor/ligand of megadock_b200.synth, seed 1000 -- at FFT N = 128,
the 54,000-rotation set, t = 3.  Writes, next to this script:

  bench_n128_D_t3.out   the reference's .out for
                        "-R bench_r.pdb -L bench_l.pdb -F 128 -t 3 -D -N 2000"
                        (relative paths, so the header names the files only),
                        MD_SHIM_FFT=fp32 (the stand-in for FFTW's float path);
                        src/docking.cpp:399-453 writes it.
  bench_n128_D_t3_rot.npz
                        per-rotation top-3 of every 15th rotation of the set
                        (3,600 rotations spread over all 54,000), from the
                        reference's CPU chain for one rotation
                        (src/docking.cpp:262-307 -> src/fft_process.cpp:399-458):
                          rot      int32 [R]          rotation index
                          score32  float32 [R, 3]     FP32 FFT (shim fp32)
                          cell32   int32 [R, 3, 3]    (i, j, k) of each record
                          score64  float32 [R, 3]     FP64 FFT of the same float
                          cell64   int32 [R, 3, 3]    grids (shim fp64)

Usage:  python tests/golden/make_goldens.py [--procs P] [--skip-out]
About 30 CPU-minutes on 8 cores (the .out is most of it).
"""
from __future__ import annotations

import argparse
import multiprocessing as mp
import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

N_REC, N_LIG, SEED = 500, 250, 1000
FLAGS = ["-F", "128", "-t", "3", "-D"]
OUT_NAME = "bench_n128_D_t3.out"
ROT_NAME = "bench_n128_D_t3_rot.npz"
ROT_STRIDE = 15
N_ROT = 54000
T = 3

_sess = None


def _init(workdir, fft):
    global _sess
    os.chdir(workdir)
    from oracle.ref import RefSession
    _sess = RefSession(["-R", "bench_r.pdb", "-L", "bench_l.pdb", *FLAGS], fft=fft)
    _sess.rec_init()


def _dock(rots):
    out = []
    for r in rots:
        s, idx = _sess.dock_rotation(int(r))
        out.append((int(r), s.copy(), idx[:, 1:].copy()))
    return out


def per_rotation(workdir, fft, procs):
    rots = np.arange(0, N_ROT, ROT_STRIDE, dtype=np.int32)
    chunks = [rots[i::procs * 4] for i in range(procs * 4)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs, initializer=_init, initargs=(workdir, fft)) as pool:
        res = [x for part in pool.map(_dock, chunks) for x in part]
    res.sort(key=lambda x: x[0])
    score = np.stack([x[1] for x in res]).astype(np.float32)
    cell = np.stack([x[2] for x in res]).astype(np.int32)
    assert [x[0] for x in res] == rots.tolist()
    return rots, score, cell


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--procs", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--skip-out", action="store_true")
    args = ap.parse_args()
    from megadock_b200 import synth
    from oracle import ref
    if not ref.available():
        raise SystemExit("oracle/_ref is not built (make -C oracle)")
    work = tempfile.mkdtemp(prefix="md_golden_")
    try:
        synth.write_pair(work, N_REC, N_LIG, SEED, stem="bench")
        rots, s32, c32 = per_rotation(work, "fp32", args.procs)
        _, s64, c64 = per_rotation(work, "fp64", args.procs)
        np.savez_compressed(HERE / ROT_NAME, rot=rots, score32=s32, cell32=c32, score64=s64, cell64=c64)
        print(f"wrote {ROT_NAME}: {len(rots)} rotations")
        if not args.skip_out:
            env = dict(os.environ, OMP_NUM_THREADS=str(args.procs), MD_SHIM_FFT="fp32")
            res = subprocess.run([str(ref.REF_BIN), "-R", "bench_r.pdb", "-L", "bench_l.pdb", *FLAGS, "-N", "2000",
                                  "-o", "ref.out"], cwd=work, env=env, capture_output=True, text=True)
            if res.returncode != 0:
                raise SystemExit(res.stderr[-2000:])
            shutil.copy(os.path.join(work, "ref.out"), HERE / OUT_NAME)
            print(f"wrote {OUT_NAME}")
    finally:
        shutil.rmtree(work, ignore_errors=True)


if __name__ == "__main__":
    main()
