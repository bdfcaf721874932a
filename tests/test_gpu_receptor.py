"""Receptor grids on the GPU (md_receptor_build) are bit-exact with the host
restatement of Receptor::rpscace + Receptor::electro (itself pinned to the
reference in test_host_parity.py) across sizes, grid widths and the -a, -d,
-e values, and give the same R^ as md_receptor_fft of the host grids."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(pairs, name, extra):
    from megadock_b200 import FFTProcess, Job
    rp, lp = pairs[name]
    job = Job(["-R", rp, "-L", lp, *extra])
    fp = FFTProcess(0)
    fp.alloc_array(job.nf1, job.grid_width, job.grid_coord())
    xyz, rad, q, ace = job.receptor_atoms()
    rc, _ = job.centers()
    xyz_c = (xyz.reshape(-1, 3) - np.asarray(rc, np.float32)).astype(np.float32)
    return job, fp, xyz_c, rad, q, ace


@pytest.mark.parametrize("name,extra,core,acer,elec", [
    ("c0", ("-F", "96"), -45.0, 1.0, 1.0),
    ("c1", ("-F", "128"), -45.0, 1.0, 1.0),
    ("small", ("-F", "64", "-a", "-20", "-d", "0.5", "-e", "0.06"), -20.0, 0.5, 0.06),
    ("small", ("-F", "96", "-v", "0.9"), -45.0, 1.0, 1.0),
    ("small", ("-F", "48", "-v", "2.0", "-d", "0"), -45.0, 0.0, 1.0),
    ("c0", ("-F", "160", "-e", "2.5"), -45.0, 1.0, 2.5),
    ("c0", ("-F", "154"), -45.0, 1.0, 1.0),
    ("c0", ("-F", "224"), -45.0, 1.0, 1.0),
    # ng1 above 112: the sweep's row masks (3 words) in global memory
    ("c0", ("-F", "240"), -45.0, 1.0, 1.0),
    ("c1", ("-F", "256", "-v", "0.9", "-e", "0.06"), -45.0, 1.0, 0.06),
    ("c0", ("-F", "320", "-v", "0.6"), -45.0, 1.0, 1.0),
    ("c0", ("-F", "400", "-v", "0.45"), -45.0, 1.0, 1.0),   # 4 mask words
])
def test_device_receptor_grids_bit_exact(built, gpu, pairs, name, extra, core, acer, elec):
    job, fp, xyz_c, rad, q, ace = _case(pairs, name, extra)
    hr, hi = job.receptor_grids()
    dr, di = fp.receptor_build(xyz_c, rad, q, ace, core, acer, elec, make_receptor=False, return_grids=True)
    assert np.array_equal(dr, hr), f"{(dr != hr).sum()} real cells differ"
    assert np.array_equal(di, hi), f"{(di != hi).sum()} field cells differ"


def test_device_receptor_spectrum_equals_host_path(built, gpu, pairs):
    job, fp, xyz_c, rad, q, ace = _case(pairs, "c0", ("-F", "96"))
    hr, hi = job.receptor_grids()
    fp.receptor_fft(hr, hi)
    want = fp.receptor_spectrum()
    fp.receptor_build(xyz_c, rad, q, ace, make_receptor=True)
    got = fp.receptor_spectrum()
    assert np.array_equal(got, want)
