"""Planted complexes on the CPU: the native pose (set rotation + grid
translation) restores the planted ligand exactly (C-alpha RMSD ~0), other
poses do not, and the per-residue-type receptor field grids add up to the
receptor's electrostatic grid."""
import numpy as np


def test_native_pose_restores_planted_ligand(built, tmp_path):
    from megadock_b200 import Job, POSE_DTYPE, rotation_matrices, synth
    from megadock_b200.fit import pose_rmsd
    pc = synth.plant_complex(str(tmp_path), 60, 30, 4100, rotation_set=360)
    job = Job(["-R", pc.rec_pdb, "-L", pc.lig_pdb, "-F", "96", "-r", "360"])
    mats = rotation_matrices(job.rotation_angles())
    rc, lc = [np.asarray(c, np.float64) for c in job.centers()]
    poses = np.zeros(3, POSE_DTYPE)
    poses["rot"] = [pc.rot_index, pc.rot_index, (pc.rot_index + 1) % 360]
    for p in range(3):
        poses[p]["i"], poses[p]["j"], poses[p]["k"] = np.asarray(pc.shift) % job.nf1
    poses[1]["i"] = (poses[1]["i"] + 5) % job.nf1
    r = pose_rmsd(poses, mats, pc.lig_file_ca, lc, rc, pc.native_ca, job.nf1, job.grid_width)
    assert r[0] < 1e-3
    assert abs(r[1] - 5 * job.grid_width) < 1e-3
    assert r[2] > 0.5
    # the planted ligand touches the receptor: closest heavy atoms about 4 A apart
    rec = job.receptor_atoms()[0].reshape(-1, 3)
    d = np.sqrt(((pc.native_ca[:, None, :] - rec[None]) ** 2).sum(-1)).min()
    assert d < 8.0


def test_receptor_field_groups_sum_to_grid(built, pairs):
    from megadock_b200 import Job
    from megadock_b200.fit import RESIDUES, residue_codes
    rp, lp = pairs["small"]
    job = Job(["-R", rp, "-L", lp, "-F", "64", "-r", "24"])
    codes = residue_codes(rp)
    assert len(codes) == job.na_rec
    U = job.receptor_elec_groups(codes, len(RESIDUES) + 1)
    _, ri = job.receptor_grids()
    tot = U.astype(np.float64).sum(0)
    assert np.allclose(tot, ri, rtol=1e-5, atol=1e-4 * np.abs(ri).max())
    # a single group holding every atom reproduces the grid bit for bit
    one = job.receptor_elec_groups(np.zeros(job.na_rec, np.int32), 1)
    assert np.array_equal(one[0], ri)


def test_pose_rmsd_closed_form_matches_direct():
    from megadock_b200 import POSE_DTYPE
    from megadock_b200.fit import pose_rmsd
    rng = np.random.default_rng(5)
    q, _ = np.linalg.qr(rng.standard_normal((40, 3, 3)))
    mats = q.reshape(40, 9).astype(np.float32)
    ca = rng.standard_normal((57, 3)) * 10 + 3
    lc, rc = np.array([1.0, -2.0, 0.5]), np.array([4.0, 4.0, -1.0])
    nat = rng.standard_normal((57, 3)) * 10
    poses = np.zeros(200, POSE_DTYPE)
    poses["rot"] = rng.integers(0, 40, 200)
    for f in ("i", "j", "k"):
        poses[f] = rng.integers(0, 96, 200)
    got = pose_rmsd(poses, mats, ca, lc, rc, nat, 96, 1.2)
    t = np.stack([poses["i"], poses["j"], poses["k"]], -1)
    t = np.where(t >= 48, t - 96, t)
    M = mats.astype(np.float64)[poses["rot"]].reshape(-1, 3, 3)
    placed = np.einsum("pij,aj->pai", M, ca - lc) - t[:, None, :] * 1.2 + rc
    want = np.sqrt(((placed - nat) ** 2).sum(-1).mean(-1))
    assert np.allclose(got, want, rtol=1e-9, atol=1e-9)
