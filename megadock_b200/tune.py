"""Autotuner for the batched form: rotations per launch.

The batched pipeline's cost per rotation falls as more rotations share a
launch (fuller grids, fewer launches) until the per-launch intermediates stop
fitting in L2.  ``autotune_batch`` times a sample of rotations at each
candidate size with the library's per-stage CUDA events (md_dock_profile) and
returns the fastest.  Results are cached per (N, t, sample) in-process.
"""
from __future__ import annotations

_cache: dict = {}

CANDIDATES = (4, 8, 16, 24, 32, 48, 64)


def autotune_batch(fp, d_rotmat: int, d_out: int, t: int, sample: int = 1536, candidates=CANDIDATES) -> int:
    key = (fp.num_fft, t, sample, tuple(candidates))
    if key in _cache:
        return _cache[key]
    best, best_ms = candidates[0], float("inf")
    for b in candidates:
        fp.set_batch(b)
        fp.dock_profile(d_rotmat, 0, min(sample, 2 * b), t, d_out)   # allocate + warm
        ms, _ = fp.dock_profile(d_rotmat, 0, sample, t, d_out)
        total = float(ms.sum())
        if total < best_ms:
            best, best_ms = b, total
    fp.set_batch(best)
    _cache[key] = best
    return best
