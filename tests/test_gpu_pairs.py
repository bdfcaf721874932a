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
