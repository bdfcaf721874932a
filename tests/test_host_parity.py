"""Host side of the drop-in contract against the reference itself (CPU).

Command line, tables, PDB reading, grid sizing, grid coordinates, centres and
the receptor grids (src/receptor.cpp) must equal MEGADOCK's bit for bit.
"""
import numpy as np
import pytest

from conftest import needs_ref


def _args(pairs, name, *extra):
    rp, lp = pairs[name]
    return ["-R", rp, "-L", lp, *extra]


CASES = [
    ("c0", ("-F", "96", "-e", "0.06", "-r", "24")),
    ("c0", ("-r", "24")),                       # automatic grid size (11-smooth table)
    ("c0", ("-r", "24", "-l", "7", "-v", "1.0")),
    ("c1", ("-F", "128", "-t", "3", "-r", "24")),
    ("small", ("-F", "64", "-a", "-30", "-d", "0.5", "-r", "24")),
    ("small", ("-F", "64", "-f", "2", "-r", "24")),
]


@needs_ref
@pytest.mark.parametrize("name,extra", CASES)
def test_receptor_grids_bit_exact(built, pairs, name, extra):
    from megadock_b200 import Job
    from oracle.ref import RefSession
    args = _args(pairs, name, *extra)
    job = Job(args)
    ref = RefSession(args)
    assert (job.ng1, job.nf1, job.na_rec, job.na_lig, job.n_rot, job.t) == \
        (ref.ng1, ref.nf1, ref.na_rec, ref.na_lig, ref.n_rot, ref.t)
    assert np.array_equal(job.grid_coord(), ref.grid_coord())
    for a, b in zip(job.centers(), ref.centers()):
        assert np.array_equal(a, b)
    jr, ji = job.receptor_grids()
    rr, ri = ref.receptor_grids()
    assert np.array_equal(jr, rr)
    assert np.array_equal(ji, ri)
    _, lrad, lq = job.ligand_atoms()
    _, rrad, rq, _ = ref.atoms(1)
    assert np.array_equal(lrad, rrad) and np.array_equal(lq, rq)
    _, jrad, jq, jace = job.receptor_atoms()
    _, rrad, rq, race = ref.atoms(0)
    assert np.array_equal(jrad, rrad) and np.array_equal(jq, rq) and np.array_equal(jace, race)


@needs_ref
@pytest.mark.parametrize("nset", [1, 3, 24, 360, 3600, 54000])
def test_rotation_sets_and_matrices(built, pairs, nset):
    """Every rotation set equals the reference's, and the rotated ligand
    coordinates from md_rotation_matrix equal Docking::ligand_rotationz's."""
    from megadock_b200 import Job, rotation_matrix
    from oracle import oracle as O
    from oracle.ref import RefSession
    args = _args(pairs, "small", "-F", "64", "-r", str(nset))
    job = Job(args)
    ref = RefSession(args)
    ang = job.rotation_angles()
    assert ang.shape == (nset, 3)
    step = max(1, nset // 200)
    xyz, _, _ = job.ligand_atoms()
    for r in range(0, nset, step):
        assert np.array_equal(ang[r], ref.angles(r))
        rx, _, _ = ref.ligand_grids(r)
        assert np.array_equal(O.rotate(xyz, rotation_matrix(ang[r])), rx)


def test_default_output_name_and_clamp(built, pairs):
    from megadock_b200 import Job
    job = Job(_args(pairs, "small", "-F", "64", "-r", "3", "-t", "2"))
    assert job.out_file == "small_r-small_l.out"
    assert job.n_out == 6            # 3 rotations x t=2 < 2000
    job = Job(_args(pairs, "small", "-F", "64", "-r", "24", "-N", "5", "-o", "x.out"))
    assert job.out_file == "x.out" and job.n_out == 5


@pytest.mark.parametrize("extra,code", [
    (("-L", "x.pdb"), 6),                                   # no receptor
    (("-R", "a.pdb", "-L", "b.pdb", "-r", "7"), 1),         # unsupported rotation set
    (("-R", "a.pdb", "-L", "b.pdb", "-f", "1", "-e", "2"), 6),
    (("-R", "a.pdb", "-L", "b.pdb", "-e", "2", "-f", "1"), 6),
    (("-R", "a.pdb", "-L", "b.pdb", "-T", "0"), 6),
    (("-R", "a.pdb", "-L", "b.pdb", "-y", "1"), 6),
    (("-R", "/nonexistent.pdb", "-L", "b.pdb"), 5),
])
def test_command_line_errors(built, extra, code):
    from megadock_b200 import Job, MdError
    with pytest.raises(MdError) as e:
        Job(list(extra))
    assert e.value.code == code


def test_grid_too_small_is_an_error(built, pairs):
    from megadock_b200 import Job, MdError
    with pytest.raises(MdError) as e:
        Job(_args(pairs, "c1", "-F", "64", "-r", "1"))
    assert e.value.code == 4 and "too big" in str(e.value)


def test_bad_pdb_record_is_an_error(built, tmp_path, pairs):
    from megadock_b200 import Job, MdError
    bad = tmp_path / "bad.pdb"
    bad.write_text("ATOM      1  CA  ALA A   1       1.000   2.000\n")
    with pytest.raises(MdError):
        Job(["-R", str(bad), "-L", pairs["small"][1], "-F", "64", "-r", "1"])


def test_hydrogen_lines_skipped(built, tmp_path, pairs):
    from megadock_b200 import Job
    src = open(pairs["small"][1]).read().splitlines()
    atoms = [l for l in src if l.startswith("ATOM")]
    h = atoms[0][:76] + " H  "
    p = tmp_path / "h.pdb"
    p.write_text("\n".join([h] + src) + "\n")
    a = Job(["-R", pairs["small"][0], "-L", str(p), "-F", "64", "-r", "1"])
    b = Job(["-R", pairs["small"][0], "-L", pairs["small"][1], "-F", "64", "-r", "1"])
    assert a.na_lig == b.na_lig
