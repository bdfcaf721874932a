"""Device pipeline parity (GPU).  Calls go through the C ABI.

  * voxel grids: bit-exact with the oracle restatement (itself pinned to the
    reference in test_oracle.py) and, where built, with the reference itself;
  * receptor spectrum: vs numpy FP64, relative max error < 2e-6;
  * per-rotation top-t: scores within 1e-4 relative of the FP64 oracle
    (|d| <= 1e-4 * |s| + 1e-3); translation indices equal, or, at a near tie,
    the oracle's score at the device's index is within the same tolerance;
  * the batched form (rotations per launch > 1, one CUDA graph) returns the
    same records as the plain form, bit for bit.
"""
import numpy as np
import pytest

from conftest import needs_ref

pytestmark = pytest.mark.gpu

RTOL = 1e-4
ATOL = 1e-3


def _args(pairs, name, *extra):
    rp, lp = pairs[name]
    return ["-R", rp, "-L", lp, *extra]


def _setup(pairs, name, *extra):
    from megadock_b200 import FFTProcess, Job
    job = Job(_args(pairs, name, *extra))
    fp = FFTProcess(0)
    fp.alloc_array(job.nf1, job.grid_width, job.grid_coord())
    rr, ri = job.receptor_grids()
    fp.receptor_fft(rr, ri)
    xyz, rad, q = job.ligand_atoms()
    fp.ligand_data_transfer_gpu(xyz, rad, q, job.lig_core)
    return job, fp


@pytest.mark.parametrize("name,extra", [
    ("c0", ("-F", "96", "-r", "3600")),
    ("c0", ("-F", "96", "-b", "2.5", "-r", "360")),
    ("c1", ("-F", "128", "-t", "3", "-r", "3600")),
    ("small", ("-F", "96", "-v", "0.9", "-r", "360")),
    ("small", ("-F", "80", "-r", "360")),
    ("small", ("-F", "160", "-r", "24")),
    ("small", ("-F", "44", "-v", "2.5", "-r", "24")),
    ("small", ("-F", "140", "-r", "24")),
    ("small", ("-F", "50", "-v", "2.5", "-r", "24")),
    ("small", ("-F", "154", "-r", "24")),
    ("small", ("-F", "162", "-r", "24")),
    ("small", ("-F", "224", "-r", "24")),
    # staged sizes (row and column launches)
    ("small", ("-F", "256", "-r", "24")),
    ("small", ("-F", "250", "-r", "24")),
    ("c0", ("-F", "320", "-v", "0.9", "-r", "24")),
    ("c0", ("-F", "400", "-v", "0.75", "-r", "24")),   # class planes in dynamic shared memory
    ("c0", ("-F", "256", "-b", "2.5", "-r", "24")),     # general core value, staged rows
])
def test_device_voxels_bit_exact(built, gpu, pairs, name, extra):
    from megadock_b200 import rotation_matrix
    from oracle import oracle as O
    job, fp = _setup(pairs, name, *extra)
    xyz, rad, q = job.ligand_atoms()
    gc = job.grid_coord()
    ang = job.rotation_angles()
    for r in range(0, job.n_rot, max(1, job.n_rot // 50)):
        m = rotation_matrix(ang[r])
        dr, di = fp.ligand_voxels(m)
        gr, gi = O.ligand_grids(O.rotate(xyz, m), rad, q, job.ng1, job.grid_width, gc, job.lig_core)
        assert np.array_equal(dr, gr), f"rotation {r}: {(dr != gr).sum()} real cells differ"
        assert np.array_equal(di, gi), f"rotation {r}: {(di != gi).sum()} charge cells differ"


@needs_ref
def test_device_voxels_vs_reference(built, gpu, pairs):
    from megadock_b200 import rotation_matrix
    from oracle.ref import RefSession
    args = ("-F", "128", "-t", "3", "-r", "54000")
    job, fp = _setup(pairs, "c1", *args)
    ref = RefSession(_args(pairs, "c1", *args))
    ang = job.rotation_angles()
    for r in range(0, 54000, 2700):
        dr, di = fp.ligand_voxels(rotation_matrix(ang[r]))
        _, rr, ri = ref.ligand_grids(r)
        assert np.array_equal(dr, rr) and np.array_equal(di, ri), r


@pytest.mark.parametrize("name,extra", [("c0", ("-F", "96",)), ("c1", ("-F", "128",)), ("small", ("-F", "160",)),
                                        ("small", ("-F", "80",)), ("small", ("-F", "112",)),
                                        ("small", ("-F", "48", "-v", "2.0")), ("small", ("-F", "88")),
                                        ("small", ("-F", "132")), ("small", ("-F", "90")), ("small", ("-F", "154")),
                                        ("small", ("-F", "192")), ("small", ("-F", "224")),
                                        ("small", ("-F", "240")), ("small", ("-F", "256")),
                                        ("small", ("-F", "270")), ("c0", ("-F", "320", "-v", "0.9"))])
def test_receptor_spectrum(built, gpu, pairs, name, extra):
    from oracle import oracle as O
    job, fp = _setup(pairs, name, *extra, "-r", "1")
    rr, ri = job.receptor_grids()
    want = O.receptor_spectrum(rr, ri, job.nf1, "fp64")
    got = fp.receptor_spectrum()
    err = np.abs(got - want).max() / np.abs(want).max()
    assert err < 2e-6, err


def _check_rotation(got, rhat, job, r, t, m):
    from oracle import oracle as O
    xyz, rad, q = job.ligand_atoms()
    gr, gi = O.ligand_grids(O.rotate(xyz, m), rad, q, job.ng1, job.grid_width, job.grid_coord(), job.lig_core)
    raw = O.raw_scores(rhat, gr, gi, "fp64")
    s, idx = O.score_sort(raw, t)
    nf = job.nf1
    nf3 = float(nf ** 3)
    errs, same = [], 0
    for k in range(t):
        g = got[k]
        assert g["rot"] == r
        assert abs(g["score"] - s[k]) <= RTOL * abs(s[k]) + ATOL, (r, k, g["score"], s[k])
        errs.append(abs(float(g["score"]) - float(s[k])) / max(abs(float(s[k])), 1e-30))
        gi_ = (g["i"], g["j"], g["k"])
        if tuple(idx[k]) != gi_:
            # near tie: the oracle's score at the device's cell must be as good
            alt = raw[gi_] / nf3
            assert abs(alt - s[k]) <= RTOL * abs(s[k]) + ATOL, (r, k, gi_, tuple(idx[k]), alt, s[k])
        else:
            same += 1
    return errs, same


@pytest.mark.parametrize("name,extra,t,nchk", [
    ("c0", ("-F", "96", "-e", "0.06", "-r", "3600"), 1, 40),
    ("c1", ("-F", "128", "-r", "54000"), 3, 12),
    ("small", ("-F", "64", "-r", "360"), 5, 30),
    ("small", ("-F", "160", "-r", "24"), 2, 4),
    ("small", ("-F", "32", "-v", "3.0", "-r", "24"), 2, 8),
    ("small", ("-F", "48", "-v", "2.0", "-r", "24"), 1, 8),
    ("small", ("-F", "80", "-r", "360"), 4, 10),
    ("small", ("-F", "112", "-r", "24"), 1, 6),
    ("small", ("-F", "120", "-r", "24"), 17, 3),
    ("small", ("-F", "144", "-r", "24"), 3, 4),
    ("small", ("-F", "36", "-v", "3.0", "-r", "24"), 2, 4),
    ("small", ("-F", "40", "-v", "3.0", "-r", "24"), 1, 4),
    ("small", ("-F", "44", "-v", "2.5", "-r", "24"), 3, 4),
    ("small", ("-F", "56", "-v", "2.0", "-r", "24"), 2, 4),
    ("small", ("-F", "60", "-v", "2.0", "-r", "24"), 2, 4),
    ("small", ("-F", "84", "-r", "24"), 3, 4),
    ("small", ("-F", "88", "-r", "24"), 2, 4),
    ("small", ("-F", "132", "-r", "24"), 3, 3),
    ("small", ("-F", "140", "-r", "24"), 2, 3),
    ("small", ("-F", "42", "-v", "3.0", "-r", "24"), 2, 4),
    ("small", ("-F", "50", "-v", "2.5", "-r", "24"), 3, 4),
    ("small", ("-F", "54", "-v", "2.0", "-r", "24"), 1, 4),
    ("small", ("-F", "66", "-r", "24"), 2, 4),
    ("small", ("-F", "70", "-r", "24"), 3, 4),
    ("small", ("-F", "90", "-r", "24"), 2, 4),
    ("small", ("-F", "98", "-r", "24"), 1, 4),
    ("small", ("-F", "110", "-r", "24"), 3, 3),
    ("small", ("-F", "126", "-r", "24"), 2, 3),
    ("small", ("-F", "150", "-r", "24"), 2, 3),
    ("small", ("-F", "154", "-r", "24"), 3, 3),
    ("small", ("-F", "162", "-r", "24"), 2, 2),
    ("small", ("-F", "168", "-r", "24"), 1, 2),
    ("small", ("-F", "176", "-r", "24"), 3, 2),
    ("small", ("-F", "192", "-r", "24"), 2, 2),
    ("small", ("-F", "210", "-r", "24"), 1, 2),
    ("small", ("-F", "224", "-r", "24"), 3, 2),
    ("small", ("-F", "72", "-r", "24"), 2, 3),
    ("small", ("-F", "100", "-r", "24"), 3, 3),
    ("small", ("-F", "108", "-r", "24"), 1, 3),
    ("small", ("-F", "180", "-r", "24"), 2, 2),
    ("small", ("-F", "196", "-r", "24"), 1, 2),
    ("small", ("-F", "198", "-r", "24"), 3, 2),
    ("small", ("-F", "200", "-r", "24"), 2, 2),
    ("small", ("-F", "216", "-r", "24"), 1, 2),
    ("small", ("-F", "220", "-r", "24"), 2, 2),
    # staged sizes above 224 (the default grid table up to ng1 = 160)
    ("small", ("-F", "240", "-r", "24"), 3, 2),
    ("small", ("-F", "242", "-r", "24"), 1, 1),
    ("small", ("-F", "250", "-r", "24"), 2, 1),
    ("small", ("-F", "252", "-r", "24"), 3, 1),
    ("small", ("-F", "256", "-r", "24"), 2, 2),
    ("small", ("-F", "256", "-r", "24"), 20, 1),
    ("small", ("-F", "264", "-r", "24"), 1, 1),
    ("small", ("-F", "270", "-r", "24"), 3, 1),
    ("small", ("-F", "280", "-r", "24"), 2, 1),
    ("c0", ("-F", "288", "-r", "24"), 3, 1),
    ("small", ("-F", "294", "-r", "24"), 1, 1),
    ("small", ("-F", "300", "-r", "24"), 2, 1),
    ("small", ("-F", "308", "-r", "24"), 3, 1),
    ("c0", ("-F", "320", "-v", "0.9", "-r", "24"), 3, 2),
    ("c0", ("-F", "400", "-v", "0.75", "-r", "24"), 2, 1),
    # ng1 of the default table in (160, 220]: odd ng1 (unpruned), pruned, the largest
    ("c0", ("-F", "330", "-v", "0.9", "-r", "24"), 2, 1),
    ("c0", ("-F", "384", "-v", "0.8", "-r", "24"), 3, 1),
    ("c0", ("-F", "440", "-v", "0.7", "-r", "24"), 1, 1),
    # ng1 in (220, 256]: odd ng1 (unpruned), 16-line x tiles for a 32-line request, the largest
    ("c0", ("-F", "486", "-v", "0.6", "-r", "24"), 2, 1),
    ("c0", ("-F", "512", "-v", "0.6", "-r", "24"), 3, 1),
    ("c0", ("-F", "256", "-b", "2.5", "-e", "0.06", "-r", "24"), 3, 1),
])
def test_dock_matches_fp64_oracle(built, gpu, pairs, name, extra, t, nchk):
    from megadock_b200 import rotation_matrices
    from oracle import oracle as O
    job, fp = _setup(pairs, name, *extra, "-t", str(t))
    rr, ri = job.receptor_grids()
    rhat = O.receptor_spectrum(rr, ri, job.nf1, "fp64")
    ang = job.rotation_angles()
    sel = np.linspace(0, job.n_rot - 1, nchk).astype(int)
    mats = rotation_matrices(ang[sel])
    got = fp.cuda_fft(mats, t=t, first_rot=0)
    errs, same = [], 0
    for n, r in enumerate(sel):
        g = got[n * t:(n + 1) * t].copy()
        g["rot"] = r
        e, k = _check_rotation(g, rhat, job, r, t, mats[n])
        errs += e
        same += k
    print(f"\nN={job.nf1} t={t}: {len(errs)} poses, max |device - FP64| / |FP64| = {max(errs):.2e}, "
          f"median {np.median(errs):.2e}; cell equal to the FP64 argmax for {same} of {len(errs)}")


@needs_ref
def test_dock_matches_reference_fp32(built, gpu, pairs):
    from megadock_b200 import rotation_matrices
    from oracle.ref import RefSession
    args = ("-F", "96", "-e", "0.06", "-r", "360", "-t", "2")
    job, fp = _setup(pairs, "c0", *args)
    ref = RefSession(_args(pairs, "c0", *args))
    ang = job.rotation_angles()
    got = fp.cuda_fft(rotation_matrices(ang[:8]), t=2)
    errs = []
    for r in range(8):
        s, idx = ref.dock_rotation(r)
        g = got[2 * r:2 * r + 2]
        np.testing.assert_allclose(g["score"], s, rtol=RTOL, atol=ATOL)
        errs += list(np.abs(g["score"].astype(np.float64) - s) / np.maximum(np.abs(s), 1e-30))
    print(f"\nvs the reference's FP32 path (project FFT shim): max relative error {max(errs):.2e}")


def test_xline_tiles_bit_identical(built, gpu, pairs):
    """8-, 16- and 32-line tiles of the x-line kernel compute the same lines."""
    from megadock_b200 import rotation_matrices
    for name, extra in (("c0", ("-F", "96", "-r", "360")), ("small", ("-F", "100", "-r", "360"))):
        job, fp = _setup(pairs, name, *extra)
        mats = rotation_matrices(job.rotation_angles()[:48])
        fp.set_batch(16)
        a = fp.cuda_fft(mats, t=3).copy()
        for tile in (16, 8):
            fp.set_tile(tile)
            b = fp.cuda_fft(mats, t=3).copy()
            assert np.array_equal(a, b), (name, tile)


@pytest.mark.parametrize("t", [1, 3, 17])
def test_n128_register_fold_forms_match_fp64_oracle(built, gpu, pairs, t):
    """N=128 with 16-line x tiles runs the register-fold x-line kernel and the
    plane kernel's fold-in-ky-pass form with warp-owned z rows (the bench's
    launch shape): its records match the FP64 oracle for one (t=1), four
    (t=3) and two passes of sixteen (t=17) selections per plane, the batched
    graph equals the plain form bit for bit, and the 32-line tiles (the
    two-phase fold kernel) agree within the tolerance."""
    from megadock_b200 import rotation_matrices
    from oracle import oracle as O
    job, fp = _setup(pairs, "small", "-F", "128", "-r", "360", "-t", str(t))
    rr, ri = job.receptor_grids()
    rhat = O.receptor_spectrum(rr, ri, job.nf1, "fp64")
    sel = np.array([0, 131, 287])
    mats_all = rotation_matrices(job.rotation_angles()[:20])
    fp.set_tile(16)
    plain = fp.cuda_fft(mats_all, t=t).copy()
    fp.set_batch(8)
    batched = fp.cuda_fft(mats_all, t=t).copy()
    assert np.array_equal(plain, batched)
    fp.set_tile(32)
    other = fp.cuda_fft(mats_all, t=t).copy()
    s0, s1 = plain["score"].astype(np.float64), other["score"].astype(np.float64)
    assert np.all(np.abs(s1 - s0) <= 2 * (RTOL * np.abs(s0) + ATOL))
    fp.set_tile(16)
    mats = rotation_matrices(job.rotation_angles()[sel])
    got = fp.cuda_fft(mats, t=t).copy()
    for n, r in enumerate(sel):
        g = got[n * t:(n + 1) * t].copy()
        g["rot"] = r
        _check_rotation(g, rhat, job, r, t, mats[n])


def test_release_work_then_dock_again(built, gpu, pairs):
    """md_release_work frees the launch groups' buffers and graphs; the next
    call allocates them again (at another launch shape too) and returns the
    same records."""
    from megadock_b200 import rotation_matrices
    job, fp = _setup(pairs, "c0", "-F", "96", "-r", "360", "-t", "2")
    mats = rotation_matrices(job.rotation_angles()[:200])
    fp.set_batch(192)
    a = fp.cuda_fft(mats, t=2).copy()
    fp.release_work()
    b = fp.cuda_fft(mats, t=2).copy()
    fp.release_work()
    fp.set_batch(24)
    c = fp.cuda_fft(mats, t=2).copy()
    assert np.array_equal(a, b) and np.array_equal(a, c)


def test_batched_equals_plain(built, gpu, pairs):
    from megadock_b200 import rotation_matrices
    job, fp = _setup(pairs, "c0", "-F", "96", "-r", "360", "-t", "3")
    mats = rotation_matrices(job.rotation_angles()[:37])
    plain = fp.cuda_fft(mats, t=3, first_rot=100)
    for b in (4, 16):
        fp.set_batch(b)
        batched = fp.cuda_fft(mats, t=3, first_rot=100)
        assert np.array_equal(plain, batched)
        again = fp.cuda_fft(mats, t=3, first_rot=100)   # graph replay
        assert np.array_equal(plain, again)
    assert (plain["rot"].reshape(-1, 3) == (100 + np.arange(37))[:, None]).all()


@pytest.mark.parametrize("extra", [("-F", "44", "-v", "2.5"), ("-F", "84"), ("-F", "132"), ("-F", "140"),
                                   ("-F", "50", "-v", "2.5"), ("-F", "110"), ("-F", "154"), ("-F", "192"),
                                   ("-F", "224"), ("-F", "256"), ("-F", "250"), ("-F", "440")])
def test_batched_forms_at_table_sizes(built, gpu, pairs, extra):
    """The 11-smooth sizes: the batched graph (both lane counts, every tile)
    returns the plain form's records bit for bit; the other radix plans agree
    within twice the FP64 tolerance."""
    from megadock_b200 import rotation_matrices
    job, fp = _setup(pairs, "small", *extra, "-r", "360", "-t", "3")
    mats = rotation_matrices(job.rotation_angles()[:40])
    plain = fp.cuda_fft(mats, t=3).copy()
    fp.set_batch(16)
    for lanes in (2, 1):
        fp.set_lanes(lanes)
        for tile in (32, 16, 8):
            fp.set_tile(tile)
            assert np.array_equal(plain, fp.cuda_fft(mats, t=3)), (lanes, tile)
    for plan in (1, 2):
        fp.set_plan(plan)
        got = fp.cuda_fft(mats, t=3).copy()
        s0, s1 = plain["score"].astype(np.float64), got["score"].astype(np.float64)
        assert np.all(np.abs(s1 - s0) <= 2 * (RTOL * np.abs(s0) + ATOL)), plan


@pytest.mark.parametrize("extra", [("-F", "90"), ("-F", "154"), ("-F", "132"), ("-F", "224"), ("-F", "256")])
def test_direct_pose_scores_at_table_sizes(built, gpu, pairs, extra):
    """The direct-sum rescoring (md_pose_scores, the adjoint's shift
    convention) gives the docking scores at their poses: the embedding
    offset floor(N/4) is the same in both, N/2 odd or even."""
    from megadock_b200 import rotation_matrices
    job, fp = _setup(pairs, "small", *extra, "-r", "24", "-t", "1")
    mats = rotation_matrices(job.rotation_angles())
    top = fp.cuda_fft(mats, t=1).copy()
    live = top[top["score"] > 0]
    assert len(live) > 0
    s = fp.pose_scores(mats[live["rot"]], live)
    ref = live["score"].astype(np.float64)
    assert np.all(np.abs(s - ref) <= RTOL * np.abs(ref) + ATOL)


def test_zero_charge_and_single_atom(built, gpu, pairs):
    """Degenerate ligands: all charges zero, and a one-atom ligand."""
    from megadock_b200 import rotation_matrices
    from oracle import oracle as O
    job, fp = _setup(pairs, "small", "-F", "64", "-r", "24")
    xyz, rad, q = job.ligand_atoms()
    rr, ri = job.receptor_grids()
    rhat = O.receptor_spectrum(rr, ri, job.nf1, "fp64")
    mats = rotation_matrices(job.rotation_angles())
    for xyz2, rad2, q2 in ((xyz, rad, np.zeros_like(q)), (xyz[:1], rad[:1], q[:1])):
        fp.ligand_data_transfer_gpu(xyz2, rad2, q2, 1.0)
        got = fp.cuda_fft(mats[:6], t=2)
        for r in range(6):
            gr, gi = O.ligand_grids(O.rotate(xyz2, mats[r]), rad2, q2, job.ng1, job.grid_width,
                                    job.grid_coord(), 1.0)
            dr, di = fp.ligand_voxels(mats[r])
            assert np.array_equal(dr, gr) and np.array_equal(di, gi)
            raw = O.raw_scores(rhat, gr, gi, "fp64")
            s, _ = O.score_sort(raw, 2)
            np.testing.assert_allclose(got[2 * r:2 * r + 2]["score"], s, rtol=RTOL, atol=ATOL)


def test_errors_are_status_codes(built, gpu):
    from megadock_b200 import FFTProcess, MdError
    fp = FFTProcess(0)
    with pytest.raises(MdError) as e:
        fp.cuda_fft(np.zeros((1, 9), np.float32))
    assert e.value.code == 3          # no grid yet
    with pytest.raises(MdError) as e:
        fp.alloc_array(230, 1.2, np.zeros(115, np.float32))
    assert e.value.code == 4          # no kernel set for N=230
    fp.alloc_array(64, 1.2, np.zeros(32, np.float32))
    with pytest.raises(MdError) as e:
        fp.ligand_data_transfer_gpu(np.zeros((40000, 3)), np.ones(40000), np.zeros(40000))
    assert e.value.code == 4


@pytest.mark.parametrize("name,extra,t", [("c0", ("-F", "96", "-r", "360"), 1), ("c1", ("-F", "128", "-r", "360"), 3),
                                          ("small", ("-F", "100", "-r", "360"), 2),
                                          ("small", ("-F", "120", "-r", "360"), 4)])
def test_plan_variants_agree(built, gpu, pairs, name, extra, t):
    """Every radix plan of the inverse plane kernel gives the plan-0 scores
    within twice the FP64-oracle tolerance (both are FP32 FFTs of the same
    grids, each within RTOL of FP64) and the same cells away from near ties."""
    from megadock_b200 import rotation_matrices
    job, fp = _setup(pairs, name, *extra)
    mats = rotation_matrices(job.rotation_angles())
    fp.set_batch(32)
    ref = fp.cuda_fft(mats, t=t).copy()
    for plan in (1, 2):
        fp.set_plan(plan)
        got = fp.cuda_fft(mats, t=t).copy()
        s0, s1 = ref["score"].astype(np.float64), got["score"].astype(np.float64)
        assert np.all(np.abs(s1 - s0) <= 2 * (RTOL * np.abs(s0) + ATOL)), plan
        same = (ref["i"] == got["i"]) & (ref["j"] == got["j"]) & (ref["k"] == got["k"])
        assert same.mean() >= 0.98, (plan, same.mean())
    fp.set_plan(0)


def test_context_switches_between_resident_and_staged_sizes(built, gpu, pairs):
    """One context docking at N = 128, then 256 (row and column launches, a
    larger candidate buffer), then 128 again returns, each time, the records
    of a fresh context of that size (batched form, graphs rebuilt)."""
    from megadock_b200 import FFTProcess, Job, rotation_matrices
    rp, lp = pairs["small"]
    jobs = {n: Job(["-R", rp, "-L", lp, "-F", str(n), "-r", "24", "-t", "3"]) for n in (128, 256)}

    def load(fp, job):
        fp.alloc_array(job.nf1, job.grid_width, job.grid_coord())
        rr, ri = job.receptor_grids()
        fp.receptor_fft(rr, ri)
        xyz, rad, q = job.ligand_atoms()
        fp.ligand_data_transfer_gpu(xyz, rad, q, job.lig_core)

    want = {}
    for n, job in jobs.items():
        fresh = FFTProcess(0)
        load(fresh, job)
        fresh.set_batch(8)
        want[n] = fresh.cuda_fft(rotation_matrices(job.rotation_angles()), t=3).copy()
        fresh.fft_memory_free()
    fp = FFTProcess(0)
    fp.set_batch(8)
    for n in (128, 256, 128):
        load(fp, jobs[n])
        got = fp.cuda_fft(rotation_matrices(jobs[n].rotation_angles()), t=3)
        assert np.array_equal(got, want[n]), n
    fp.fft_memory_free()
