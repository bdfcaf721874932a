"""The autotuner's search on the CPU, against a stand-in context whose
per-stage times are a known function of the launch shape: it keeps the
fastest rotations-per-launch, radix plan and tile, leaves them set on the
context and answers the same size from its cache."""


class FakeContext:
    def __init__(self, num_fft, best=(32, 2, 16)):
        self.num_fft = num_fft
        self.batch, self.plan, self.tile = 1, 0, 32
        self.best = best
        self.calls = 0

    def set_batch(self, b):
        self.batch = b

    def set_plan(self, p):
        self.plan = p

    def set_tile(self, t):
        self.tile = t

    def release_work(self):
        self.released = True

    def set_lanes(self, n):
        self.lanes = n

    def dock_profile(self, d_rot, first, n, t, d_out):
        import numpy as np
        self.calls += 1
        b0, p0, t0 = self.best
        ms = 10.0 + abs(self.batch - b0) * 0.1 + (0 if self.plan == p0 else 1.0) + (0 if self.tile == t0 else 0.5)
        return np.full(5, ms / 5, np.float32), 5


def test_autotune_picks_the_fastest_shape_and_caches():
    from megadock_b200 import tune
    tune._cache.clear()
    fp = FakeContext(96, best=(32, 2, 16))
    b, p = tune.autotune(fp, 0, 0, 3, sample=256, time_graph=lambda f: 5.0 if f.lanes == 1 else 6.0)
    assert (b, p, fp.tile, fp.lanes) == (32, 2, 16, 1)
    assert (fp.batch, fp.plan, fp.tile) == (32, 2, 16)
    n = fp.calls
    fp2 = FakeContext(96, best=(8, 0, 32))
    assert tune.autotune(fp2, 0, 0, 3, sample=256) == (32, 2)   # same size: cached answer
    assert fp2.calls == 0 and (fp2.batch, fp2.plan, fp2.tile, fp2.lanes) == (32, 2, 16, 1)
    fp3 = FakeContext(128, best=(64, 0, 8))
    assert tune.autotune(fp3, 0, 0, 3, sample=256, time_graph=lambda f: 7.0 if f.lanes == 1 else 6.0) == (64, 0)
    assert fp3.tile == 8 and fp3.lanes == 2
    assert n == 2 * len(tune.CANDIDATES) + 2 * (len(tune.PLANS) - 1) + 2 * (len(tune.TILES) - 1)


def test_autotune_skips_batches_over_the_work_budget():
    from megadock_b200 import tune
    tune._cache.clear()
    fp = FakeContext(160, best=(512, 0, 32))
    per_rot = tune.work_bytes_per_rotation(160)
    assert 320 * per_rot <= tune.WORK_BUDGET < 384 * per_rot
    b, _ = tune.autotune(fp, 0, 0, 3, sample=256, time_graph=lambda f: 1.0)
    assert b == 320 and fp.released
