"""md_dock_noalloc: the allocation-free entry point (GPU).

Callers that cannot allocate device memory -- a framework whose pool allocator
owns the device's memory, a plugin that must not grow its host's footprint, a
loop where cudaMalloc/cudaFree and their device-wide synchronisation are not
allowed -- use md_dock_noalloc, which keeps its intermediates in a fixed
32 MiB static device array.  This test calls it through the C ABI with
caller-owned device buffers and checks, on two calls in a row, that its poses
match md_dock's for the same rotations, within the tolerance the parity tests
use (scores within 1e-4 relative + 1e-3; cells identical).

The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-4
ATOL = 1e-3


def _check(got, want):
    assert np.array_equal(got["rot"], want["rot"])
    np.testing.assert_allclose(got["score"], want["score"], rtol=RTOL, atol=ATOL)
    for f in ("i", "j", "k"):
        assert np.array_equal(got[f], want[f]), f


@pytest.fixture(scope="module")
def big_ligand(tmp_path_factory):
    """A pair whose ligand has close to the 32,768-atom limit."""
    from megadock_b200 import synth
    return synth.write_pair(str(tmp_path_factory.mktemp("big")), 40, 3900, 77, stem="big")


@pytest.mark.parametrize("name,extra", [("c0", ("-F", "96", "-e", "0.06", "-t", "3")),
                                        ("small", ("-F", "110", "-t", "2")), ("small", ("-F", "88", "-t", "1")),
                                        # t > 16: several top-t passes of the plane kernel per rotation
                                        ("small", ("-F", "64", "-t", "20")),
                                        ("big", ("-F", "128", "-v", "2.0", "-t", "3"))])
def test_noalloc_matches_md_dock(built, gpu, pairs, big_ligand, name, extra):
    import torch

    from megadock_b200 import POSE_DTYPE, FFTProcess, Job, lib, rotation_matrices

    rp, lp = big_ligand if name == "big" else pairs[name]
    job = Job(["-R", rp, "-L", lp, "-r", "360", *extra])
    if name == "big":
        assert 30000 < job.na_lig <= 32768, job.na_lig
    fp = FFTProcess(0)
    fp.alloc_array(job.nf1, job.grid_width, job.grid_coord())
    rr, ri = job.receptor_grids()
    fp.receptor_fft(rr, ri)
    xyz, rad, q = job.ligand_atoms()
    fp.ligand_data_transfer_gpu(xyz, rad, q, job.lig_core)
    rhat = fp.receptor_spectrum()
    mats = rotation_matrices(job.rotation_angles())

    # caller-owned device buffers (the caller's allocator, not the library's)
    dev = torch.device("cuda:0")
    d_gc = torch.from_numpy(job.grid_coord()).to(dev)
    inter = np.empty(rhat.size * 2, np.float32)
    inter[0::2] = rhat.real.reshape(-1)
    inter[1::2] = rhat.imag.reshape(-1)
    d_rhat = torch.from_numpy(inter).to(dev)
    d_xyz = torch.from_numpy(np.ascontiguousarray(xyz.reshape(-1))).to(dev)
    d_rad = torch.from_numpy(rad).to(dev)
    d_q = torch.from_numpy(q).to(dev)

    t = job.t
    for first, n in ((0, 20), (137, 25)):          # two calls in a row
        want = fp.cuda_fft(mats[first:first + n], t=t, first_rot=first)
        d_rot = torch.from_numpy(np.ascontiguousarray(mats[first:first + n])).to(dev)
        d_out = torch.zeros(n * t * 5, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        rc = lib().md_dock_noalloc(job.nf1, C.c_float(job.grid_width), C.c_void_p(d_gc.data_ptr()),
                                   C.c_void_p(d_rhat.data_ptr()), len(rad), C.c_void_p(d_xyz.data_ptr()),
                                   C.c_void_p(d_rad.data_ptr()), C.c_void_p(d_q.data_ptr()),
                                   C.c_float(job.lig_core), C.c_void_p(d_rot.data_ptr()), first, n, t,
                                   C.c_void_p(d_out.data_ptr()), None)
        assert rc == 0
        torch.cuda.synchronize()
        got = d_out.cpu().numpy().view(POSE_DTYPE)
        _check(got, want)
    fp.fft_memory_free()


def test_noalloc_rejects_oversized_requests(built, gpu):
    from megadock_b200 import lib
    dummy = C.c_void_p(16)
    # N = 160 is above nf1 = 128, the largest edge the fixed scratch array is sized for
    rc = lib().md_dock_noalloc(160, C.c_float(1.2), dummy, dummy, 10, dummy, dummy, dummy, C.c_float(1.0), dummy,
                               0, 1, 1, dummy, None)
    assert rc == 4
    # too many poses per rotation
    rc = lib().md_dock_noalloc(96, C.c_float(1.2), dummy, dummy, 10, dummy, dummy, dummy, C.c_float(1.0), dummy,
                               0, 1, 1000, dummy, None)
    assert rc == 4
