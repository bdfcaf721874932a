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
