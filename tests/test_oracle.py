"""The oracle restatement against the reference compiled from its sources (CPU).

This pins the checker used by the GPU tests: rotations, voxel grids and the
top-t scan are bit-exact with MEGADOCK's CPU code; the FFT shim and numpy's
FFT agree to float precision.
"""
import numpy as np
import pytest

from conftest import needs_ref


def _args(pairs, name, *extra):
    rp, lp = pairs[name]
    return ["-R", rp, "-L", lp, *extra]


@needs_ref
@pytest.mark.parametrize("name,extra,delta", [
    ("c0", ("-F", "96", "-r", "3600"), 1.0),
    ("c0", ("-F", "96", "-b", "2.5", "-r", "360"), 2.5),
    ("c1", ("-F", "128", "-t", "3", "-r", "360"), 1.0),
    ("small", ("-F", "96", "-v", "0.9", "-r", "360"), 1.0),
])
def test_voxel_grids_bit_exact(built, pairs, name, extra, delta):
    from megadock_b200 import Job
    from oracle import oracle as O
    from oracle.ref import RefSession
    args = _args(pairs, name, *extra)
    job = Job(args)
    ref = RefSession(args)
    xyz, rad, q = job.ligand_atoms()
    gc = job.grid_coord()
    ang = job.rotation_angles()
    for r in range(0, job.n_rot, max(1, job.n_rot // 60)):
        m = O.rotation_matrix(ang[r])
        xr = O.rotate(xyz, m)
        rx, rr, ri = ref.ligand_grids(r)
        assert np.array_equal(xr, rx)
        gr, gi = O.ligand_grids(xr, rad, q, job.ng1, job.grid_width, gc, delta)
        assert np.array_equal(gr, rr), f"rotation {r}: {(gr != rr).sum()} real cells differ"
        assert np.array_equal(gi, ri), f"rotation {r}: {(gi != ri).sum()} charge cells differ"


@needs_ref
@pytest.mark.parametrize("t", [1, 3])
def test_score_sort_matches_reference(built, pairs, t):
    """oracle_score_sort on the reference's own score grid reproduces
    FFTProcess::score_sort exactly (t = 1 and t > 1 rules)."""
    from oracle import oracle as O
    from oracle.ref import RefSession
    ref = RefSession(_args(pairs, "small", "-F", "64", "-r", "24", "-t", str(t)))
    for r in (0, 5, 17):
        s, idx = ref.dock_rotation(r)
        raw = ref.score_grid()
        s2, idx2 = O.score_sort(raw, t)
        assert np.array_equal(s, s2)
        assert np.array_equal(idx[:, 1:], idx2)
        assert (idx[:, 0] == r).all()


@needs_ref
def test_fft_shim_and_numpy_agree(built, pairs):
    """Receptor spectrum of the reference (FP32 FFT shim) vs numpy FP64."""
    from megadock_b200 import Job
    from oracle import oracle as O
    from oracle.ref import RefSession
    args = _args(pairs, "c0", "-F", "96", "-r", "1")
    job = Job(args)
    ref = RefSession(args)
    rr, ri = job.receptor_grids()
    r64 = O.receptor_spectrum(rr, ri, job.nf1, "fp64")
    r32 = ref.spectrum()
    err = np.abs(r32 - r64).max() / np.abs(r64).max()
    assert err < 2e-6, err


@needs_ref
def test_fp64_oracle_vs_reference_fp32(built, pairs):
    """Top scores of the FP64 oracle and the reference's FP32 path agree
    within 1e-4 relative; this bounds the FP32 error the device is held to."""
    from megadock_b200 import Job
    from oracle import oracle as O
    from oracle.ref import RefSession
    args = _args(pairs, "c0", "-F", "96", "-e", "0.06", "-r", "24")
    job = Job(args)
    ref = RefSession(args)
    rr, ri = job.receptor_grids()
    rhat = O.receptor_spectrum(rr, ri, job.nf1, "fp64")
    xyz, rad, q = job.ligand_atoms()
    for r in (0, 7, 23):
        s_ref, idx_ref = ref.dock_rotation(r)
        s, idx = O.dock_rotation(rhat, xyz, rad, q, job.rotation_angles()[r], job.ng1, job.grid_width,
                                 job.grid_coord(), 1)
        assert abs(s[0] - s_ref[0]) <= 1e-4 * abs(s_ref[0]) + 1e-3
