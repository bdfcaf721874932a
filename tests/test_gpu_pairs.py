"""Batched form over uneven pairs (GPU): one graph over pairs of different
FFT sizes returns, pair by pair, exactly the poses of docking each pair alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_pairs_equal_single_pair_docking(built, gpu, tmp_path):
    from megadock_b200 import FFTProcess, rotation_matrices, synth
    from megadock_b200.pairs import PairBatch
    files = [synth.write_pair(str(tmp_path), nr, nl, seed, stem=f"q{seed}")
             for nr, nl, seed in [(30, 16, 8), (120, 60, 31), (60, 40, 32), (200, 90, 33)]]
    pb = PairBatch(files, rotation_set=360, t=2, autotune=False)
    for fp, b in zip(pb.ctxs, (7, 16, 5, 32)):
        fp.set_batch(b)
    assert len(set(pb.sizes())) >= 3, pb.sizes()
    pb.run()
    got = pb.poses()
    pb.run()                                   # graph replay
    again = pb.poses()
    for p, (job, fp) in enumerate(zip(pb.jobs, pb.ctxs)):
        mats = rotation_matrices(job.rotation_angles())
        fp.set_batch(1)
        want = fp.cuda_fft(mats, t=2)
        assert np.array_equal(got[p], want), (p, pb.sizes()[p])
        assert np.array_equal(again[p], want)


def test_fft_size_choice(built, tmp_path):
    from megadock_b200 import synth
    from megadock_b200.pairs import choose_fft_size, required_ng
    rp, lp = synth.write_pair(str(tmp_path), 150, 70, 0)
    n = choose_fft_size(rp, lp)
    assert n % 4 == 0 and n // 2 >= required_ng(rp, lp)


def test_pairs_graph_follows_pair_changes(built, gpu, tmp_path):
    """A pair context whose grid width or ligand core value changes between two
    md_dock_pairs calls (same sizes, same buffers) must not replay the graph
    captured with the old values: the second call equals single-pair docking
    at the new values."""
    from megadock_b200 import Job, rotation_matrices, synth
    from megadock_b200.pairs import PairBatch
    files = [synth.write_pair(str(tmp_path), nr, nl, seed, stem=f"g{seed}")
             for nr, nl, seed in [(30, 16, 8), (60, 40, 32)]]
    pb = PairBatch(files, rotation_set=24, t=2, autotune=False)
    for fp in pb.ctxs:
        fp.set_batch(8)
    pb.run()
    before = pb.poses()
    job, fp = pb.jobs[0], pb.ctxs[0]
    rp, lp = files[0]
    moved = Job(["-R", rp, "-L", lp, "-F", str(job.nf1), "-r", "24", "-t", "2", "-v", "1.3"])
    fp.alloc_array(job.nf1, moved.grid_width, moved.grid_coord())   # same N: only the width changes
    xyz, rad, q = job.ligand_atoms()
    fp.ligand_data_transfer_gpu(xyz, rad, q, 2.5)                   # same atom count: only -b changes
    pb.run()
    after = pb.poses()
    mats = rotation_matrices(job.rotation_angles())
    fp.set_batch(1)
    want = fp.cuda_fft(mats, t=2)
    assert np.array_equal(after[0], want)
    assert not np.array_equal(after[0], before[0])
    assert np.array_equal(after[1], before[1])
