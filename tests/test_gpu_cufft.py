"""The fused pipeline against the cuFFT comparator (GPU).

The comparator computes each rotation's score grid the way the reference's
GPU path does (fft_process.cpp:502-656: C2C forward, conj(R^) L^ product,
C2C inverse, Re / nf3) with the CUDA FFT library, from the library's own
ligand grids (bit-exact with the reference's voxelization).  Both sides are
FP32, so the bound is the parity tolerance of the path:

  * receptor spectrum: max |fused - cuFFT| / max |cuFFT| < 5e-6;
  * per-rotation top-t: each fused score within 1e-4 relative (+1e-3
    absolute) of the comparator's score of the same rank, and the
    comparator's score at the fused pose's cell within the same tolerance
    of the fused score (equal cells except at near ties).
"""
import numpy as np
import pytest

from test_gpu_parity import _setup

pytestmark = pytest.mark.gpu

RTOL = 1e-4
ATOL = 1e-3


@pytest.mark.parametrize("name,extra", [("c0", ("-F", "96")), ("c1", ("-F", "128")), ("small", ("-F", "80")),
                                        ("small", ("-F", "160"))])
def test_receptor_spectrum_vs_cufft(built, gpu, pairs, name, extra):
    from megadock_b200 import cufft_check as CF
    job, fp = _setup(pairs, name, *extra, "-r", "1")
    rr, ri = job.receptor_grids()
    want = CF.receptor_spectrum(rr, ri, job.nf1).cpu().numpy()
    got = fp.receptor_spectrum()
    err = np.abs(got - want).max() / np.abs(want).max()
    print(f"\nN={job.nf1}: receptor spectrum max |fused - cuFFT| / max |cuFFT| = {err:.2e}")
    assert err < 5e-6, err


@pytest.mark.parametrize("name,extra,t,nrot", [
    ("c0", ("-F", "96", "-e", "0.06", "-r", "3600"), 1, 24),
    ("c1", ("-F", "128", "-r", "54000"), 3, 12),
    ("small", ("-F", "80", "-r", "360"), 4, 16),
    ("small", ("-F", "144", "-r", "360"), 2, 8),
])
def test_dock_vs_cufft(built, gpu, pairs, name, extra, t, nrot):
    from megadock_b200 import cufft_check as CF
    from megadock_b200 import rotation_matrices
    job, fp = _setup(pairs, name, *extra, "-t", str(t))
    rr, ri = job.receptor_grids()
    rhat = CF.receptor_spectrum(rr, ri, job.nf1)
    sel = np.linspace(0, job.n_rot - 1, nrot).astype(int)
    mats = rotation_matrices(job.rotation_angles()[sel])
    got = fp.cuda_fft(mats, t=t).reshape(nrot, t)
    vr, vi = zip(*(fp.ligand_voxels(m) for m in mats))
    errs, same = [], 0
    for b0 in range(0, nrot, 4):
        lig = CF.embed(np.stack(vr[b0:b0 + 4]), np.stack(vi[b0:b0 + 4]), job.nf1)
        sg = CF.scores(rhat, lig)
        want, want_ijk = CF.top_t(sg, t)
        g = got[b0:b0 + 4]
        cells = np.stack([g["i"], g["j"], g["k"]], axis=-1)
        at_cells = CF.cell_scores(sg, cells)
        for n in range(len(g)):
            for k in range(t):
                s_ref = float(want[n, k])
                s = float(g["score"][n, k])
                if t == 1 and s_ref <= 0.0:
                    # t = 1 keeps a running maximum that starts at 0: no
                    # positive score gives (0, cell 0)
                    assert s == 0.0, (b0 + n, s, s_ref)
                    continue
                assert abs(s - s_ref) <= RTOL * abs(s_ref) + ATOL, (b0 + n, k, s, s_ref)
                assert abs(float(at_cells[n, k]) - s) <= RTOL * abs(s) + ATOL, (b0 + n, k, cells[n, k])
                errs.append(abs(s - s_ref) / max(abs(s_ref), 1e-30))
                same += int(tuple(cells[n, k]) == tuple(want_ijk[n, k]))
    print(f"\nN={job.nf1} t={t}: {len(errs)} poses, max |fused - cuFFT| / |cuFFT| = {max(errs):.2e}; "
          f"same cell for {same} of {len(errs)}")
