"""Autotuner for the batched form: rotations per launch, radix plan and tile.

The batched pipeline's cost per rotation falls as more rotations share a
launch (fuller grids, fewer launches) until the per-launch intermediates stop
fitting in L2, and the inverse plane kernel (the largest stage) runs at
different speeds with different radix splits of its two axes (md_set_plan:
variant 0 the line plans, 1 the kz split reversed, 2 the ky split reversed),
depending on the size, and the x-line kernel works on tiles of 8, 16 or 32
kz lines per CTA (md_set_tile).  ``autotune`` times a sample of rotations with
the library's per-stage CUDA events (md_dock_profile): first every batch size
with plan 0 and 32-line tiles, then every plan at the best batch, then the
other tiles, and keeps the fastest combination.  Last it times the whole
batched graph (md_dock_device) with one and with two launch groups in flight
(md_set_lanes): the per-stage events serialise the stages, so they cannot see
how two groups' kernels share the GPU.  Batch sizes whose two work
sets would exceed WORK_BUDGET bytes are skipped, and the work buffers are
released at the end so that the next call allocates them for the chosen
batch only.  Results are cached per (N, t, sample) in-process.
"""
from __future__ import annotations

_cache: dict = {}

CANDIDATES = (4, 8, 16, 24, 32, 48, 64, 96, 128, 192, 256, 320, 384, 512)
PLANS = (0, 1, 2)
TILES = (32, 16, 8)
LANES = (2, 1)
WORK_BUDGET = 24 << 30   # of the B200's 180 GB


def work_bytes_per_rotation(n: int) -> int:
    """Device bytes one rotation of a launch group holds in the two work sets
    (spectrum planes, Hermitian half, charge lists; the small buffers
    ignored)."""
    ng = n // 2
    return 2 * (8 * ng * n * n + 8 * n * ng * n + 8 * ng ** 3)


def _time(fp, d_rotmat, d_out, t, sample, b):
    fp.set_batch(b)
    fp.dock_profile(d_rotmat, 0, min(sample, 2 * b), t, d_out)   # allocate + warm
    ms, _ = fp.dock_profile(d_rotmat, 0, sample, t, d_out)
    return float(ms.sum())


def _time_graph(fp, d_rotmat, d_out, t, sample, reps=3):
    # the context may launch on a stream of its own, so the device is
    # synchronised around the runs (a few ms of graph each)
    import time

    import torch
    fp.dock_device(d_rotmat, 0, sample, t, d_out)   # capture + warm
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        fp.dock_device(d_rotmat, 0, sample, t, d_out)
    torch.cuda.synchronize()
    return 1000.0 * (time.perf_counter() - t0)


def autotune(fp, d_rotmat: int, d_out: int, t: int, sample: int = 1536, candidates=CANDIDATES,
             plans=PLANS, tiles=TILES, lanes=LANES, time_graph=None) -> tuple[int, int]:
    """(rotations per launch, plan) for context fp; batch, plan, tile and
    lanes are left set on fp (fp.tile, fp.lanes).  time_graph(fp) -> ms
    replaces the whole-graph timing (tests)."""
    key = (fp.num_fft, t, sample, tuple(candidates), tuple(plans), tuple(tiles), tuple(lanes))
    if key in _cache:
        b, p, tl, ln = _cache[key]
        fp.set_batch(b)
        fp.set_plan(p)
        fp.set_tile(tl)
        fp.set_lanes(ln)
        return b, p
    fp.set_plan(plans[0])
    fp.set_tile(tiles[0])
    fits = [b for b in candidates if b * work_bytes_per_rotation(fp.num_fft) <= WORK_BUDGET] or [candidates[0]]
    best_b, best_ms = fits[0], float("inf")
    for b in fits:
        ms = _time(fp, d_rotmat, d_out, t, sample, b)
        if ms < best_ms:
            best_b, best_ms = b, ms
    best_p = plans[0]
    for p in plans[1:]:
        fp.set_plan(p)
        ms = _time(fp, d_rotmat, d_out, t, sample, best_b)
        if ms < best_ms:
            best_p, best_ms = p, ms
    fp.set_plan(best_p)
    best_t = tiles[0]
    for tl in tiles[1:]:
        fp.set_tile(tl)
        ms = _time(fp, d_rotmat, d_out, t, sample, best_b)
        if ms < best_ms:
            best_t, best_ms = tl, ms
    fp.set_batch(best_b)
    fp.set_tile(best_t)
    timer = time_graph or (lambda f: _time_graph(f, d_rotmat, d_out, t, sample))
    best_l, best_g = lanes[0], float("inf")
    for ln in lanes:
        fp.set_lanes(ln)
        ms = timer(fp)
        if ms < best_g:
            best_l, best_g = ln, ms
    fp.set_lanes(best_l)
    fp.release_work()
    _cache[key] = (best_b, best_p, best_t, best_l)
    return best_b, best_p


def autotune_batch(fp, d_rotmat: int, d_out: int, t: int, sample: int = 1536, candidates=CANDIDATES) -> int:
    """Rotations per launch (the plan is tuned and set on fp too)."""
    return autotune(fp, d_rotmat, d_out, t, sample, candidates)[0]
