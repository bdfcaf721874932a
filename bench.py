"""Benchmark: rotations/s of the docking hot path at 128^3, 54,000 rotations.

Workload: a synthetic receptor of 500 residues (~4,000 heavy atoms) and ligand
of 250 residues (~1,900 atoms) (megadock_b200.synth, seed 1000), FFT N = 128,
the 54,000-rotation set, top-3 poses per rotation.  One step = every rotation
of that job through the device pipeline (rotate, voxelize, forward FFT,
conj(R^) product, inverse FFT, top-t).

  value   batched form (rotations per launch > 1, one CUDA graph), inputs
          resident in HBM (rotation matrices and pose buffer on the device)
  plain   the plain form (one rotation per fused pipeline) on the same GPU
  e2e     the batched form through the C ABI with host buffers: receptor grid
          upload + receptor FFT + ligand upload + md_dock (rotation matrices in,
          poses out) every step
  roofline  dominant kernel from per-stage CUDA events (md_dock_profile on the
          launch stream), algorithmic bytes per launch / mean launch time
  cpu_baseline  the reference's own CPU program (oracle/_ref/megadock-ref,
          MEGADOCK CPU sources + project FFT shim) on this host, bounded sample

--impl reference runs only the reference's CPU program on the same workload
(bounded sample per step) and prints its line.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_FFT = 128
N_REC, N_LIG, SEED = 500, 250, 1000
T_POSES = 3
ROT_SET = 54000
METRIC = "rotations/sec at 128^3, 54k rot: batched vs plain fused, same GPU, 1e-4 tol"
REF_SAMPLE_ROT = 360
REF_GPU_SAMPLE_ROT = 3600
SCIPY_SAMPLE_ROT = 64
PLAIN_SAMPLE = 5400


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def __enter__(self):
        def run():
            q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,utilization.gpu")
            try:
                p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            except OSError:
                return
            while not self._stop.is_set():
                line = p.stdout.readline()
                if not line:
                    break
                self.rows.append([x.strip() for x in line.split(",")])
            p.terminate()

        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=3)

    def summary(self):
        load = [r for r in self.rows if len(r) >= 7 and r[6].isdigit() and int(r[6]) > 50]
        rows = load or self.rows
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if len(r) > 2 + k and r[2 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def make_inputs(tmp):
    from megadock_b200 import synth
    return synth.write_pair(tmp, N_REC, N_LIG, SEED, stem="bench")


def workload_config(rp, lp):
    """The workload's name and sizes, the same for both arms (atoms counted
    from the generated PDB records)."""
    def atoms(path):
        with open(path) as f:
            return sum(1 for line in f if line.startswith(("ATOM", "HETATM")))
    return {"workload": f"docking, {N_REC}/{N_LIG}-residue synthetic pair ({atoms(rp)}/{atoms(lp)} atoms), "
                        f"N={N_FFT}, {ROT_SET} rotations, t={T_POSES}",
            "fft": N_FFT, "rotations": ROT_SET, "t": T_POSES}


def cpu_reference(rp, lp, nrot=REF_SAMPLE_ROT):
    """Time the reference's CPU program (all host cores) on nrot rotations."""
    from oracle import ref
    cores = os.cpu_count() or 1
    env = dict(os.environ, OMP_NUM_THREADS=str(cores), MD_SHIM_FFT="fp32")
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "ref.out")
        res = subprocess.run([str(ref.REF_BIN), "-R", rp, "-L", lp, "-F", str(N_FFT), "-t", str(T_POSES), "-r",
                              str(nrot), "-o", out], capture_output=True, text=True, env=env)
    if res.returncode != 0:
        raise RuntimeError(res.stderr[-500:])
    m = re.search(r"CPU time \(docking\)\s*=\s*([0-9.]+)", res.stdout)
    secs = float(m.group(1))
    return nrot / secs, cores, secs


def cpu_production_fft(rp, lp, nrot=SCIPY_SAMPLE_ROT):
    """The same pipeline on the host cores with a production FFT library:
    voxel grids from the oracle's C restatement of the reference's CPU
    voxelizer, scipy.fft complex64 transforms (pocketfft/ducc, workers = all
    host cores), the conj(R^) product, the inverse transform and the
    reference's top-t rules, over the first nrot rotations of the job."""
    import numpy as np
    import scipy.fft as sf

    from megadock_b200 import Job, rotation_matrices
    from oracle import oracle as O
    job = Job(["-R", rp, "-L", lp, "-F", str(N_FFT), "-t", str(T_POSES), "-D"])
    rr, ri = job.receptor_grids()
    xyz, rad, q = job.ligand_atoms()
    mats = rotation_matrices(job.rotation_angles()[:nrot])
    gc = job.grid_coord()
    cores = os.cpu_count() or 1
    with sf.set_workers(cores):
        rhat = O.receptor_spectrum(rr, ri, job.nf1, "fp32")
        t0 = time.perf_counter()
        for m in mats:
            gr, gi = O.ligand_grids(O.rotate(xyz, m), rad, q, job.ng1, job.grid_width, gc, job.lig_core)
            O.score_sort(O.raw_scores(rhat, gr, gi, "fp32"), T_POSES)
        secs = time.perf_counter() - t0
    return {"value": nrot / secs, "unit": "rotations/s", "cores": cores, "kind": "port",
            "sample": f"first {nrot} rotations of the same job ({secs:.1f} s)",
            "fft": f"scipy.fft (pocketfft) complex64, workers={cores}"}


def gpu_reference(rp, lp, nrot=REF_GPU_SAMPLE_ROT):
    """Time the reference's own GPU program (oracle/_ref/megadock-gpu-ref: its
    CUDA path -- per-rotation voxelization kernels, cuFFT C2C transforms and
    the block-maximum search, src/fft_process.cpp:502-807 -- built from its
    sources for sm_100a) on nrot rotations of the same job, one host thread
    driving the one GPU.  Rate = nrot / its "CPU time (docking)" line (wall
    time of the rotation loop)."""
    from oracle import ref
    exe = ref.REF_BIN.parent / "megadock-gpu-ref"
    if not exe.exists():
        return {"unavailable": "oracle/_ref/megadock-gpu-ref was not built (needs the reference sources and cuFFT)"}
    env = dict(os.environ, OMP_NUM_THREADS="1", MD_SHIM_FFT="fp32")
    with tempfile.TemporaryDirectory() as d:
        res = subprocess.run([str(exe), "-R", rp, "-L", lp, "-F", str(N_FFT), "-t", str(T_POSES), "-r", str(nrot),
                              "-o", os.path.join(d, "gpu.out")], capture_output=True, text=True, env=env,
                             timeout=900)
    if res.returncode != 0:
        return {"error": (res.stdout + res.stderr)[-300:]}
    m = re.search(r"CPU time \(docking\)\s*=\s*([0-9.]+)", res.stdout)
    secs = float(m.group(1))
    return {"value": nrot / secs, "unit": "rotations/s", "seconds": secs,
            "sample": f"{nrot} rotations (-r {nrot}) of the same job, N={N_FFT}, t={T_POSES}",
            "what": "MEGADOCK's own GPU path (cuFFT, one host thread, one GPU), unmodified sources built for "
                    "sm_100a; its t > 1 keeps one candidate per 512-cell block"}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import ref
    with tempfile.TemporaryDirectory() as tmp:
        rp, lp = make_inputs(tmp)
        config = workload_config(rp, lp)
        if not ref.available():
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (reference compiled from its "
                                                                  "sources) was not built on this machine"}))
            return
        for _ in range(args.warmup):
            cpu_reference(rp, lp)
        rates = []
        t0 = time.perf_counter()
        for _ in range(args.steps):
            r, cores, secs = cpu_reference(rp, lp)
            rates.append(r)
        wall = time.perf_counter() - t0
    value = statistics.mean(rates)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "rotations/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * wall / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {**config, "sampled_rotations_per_step": REF_SAMPLE_ROT,
                   "rate": f"rotations/s of the {REF_SAMPLE_ROT}-rotation sample, the per-rotation cost being "
                           f"independent of the rotation count"},
        "cpu_baseline": {"value": value, "unit": "rotations/s", "cores": cores, "kind": "reference",
                         "fft": "project-written scalar FFTW-API shim (libfftw3f is not on the image)",
                         "sample": f"{REF_SAMPLE_ROT} rotations per step (MEGADOCK CPU sources + FFTW-API shim, "
                                   f"OpenMP over all host cores)"},
        "e2e": {"value": value, "unit": "rotations/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    try:
        import torch
        if torch.cuda.is_available():
            with tempfile.TemporaryDirectory() as tmp:
                rp, lp = make_inputs(tmp)
                line["reference_gpu"] = gpu_reference(rp, lp)
    except Exception as e:  # an extra comparator, never required
        line["reference_gpu"] = {"error": str(e)[:200]}
    print(json.dumps(line, default=float))


def run_profile_case(args):
    """A small batched run of the same workload for ncu: R rotations, one pass."""
    import torch

    from megadock_b200 import FFTProcess, Job, rotation_matrices
    with tempfile.TemporaryDirectory() as tmp:
        rp, lp = make_inputs(tmp)
        job = Job(["-R", rp, "-L", lp, "-F", str(args.fft or N_FFT), "-t", str(T_POSES), "-D", "-o",
                   os.path.join(tmp, "p.out")])
        mats = rotation_matrices(job.rotation_angles()[:args.profile_case])
        fp = FFTProcess(0)
        fp.alloc_array(job.nf1, job.grid_width, job.grid_coord())
        rr, ri = job.receptor_grids()
        fp.receptor_fft(rr, ri)
        xyz, rad, q = job.ligand_atoms()
        fp.ligand_data_transfer_gpu(xyz, rad, q, job.lig_core)
        fp.set_batch(args.batch or 16)
        fp.set_plan(args.plan)
        fp.set_tile(args.tile)
        d_rot = torch.from_numpy(mats).cuda()
        d_pose = torch.zeros(len(mats) * T_POSES * 5, dtype=torch.int32, device="cuda")
        fp.dock_profile(d_rot.data_ptr(), 0, len(mats), T_POSES, d_pose.data_ptr())
        torch.cuda.synchronize()
        fp.fft_memory_free()
    print("profile case done")


def run_profile_aux(args):
    """One small invocation of every auxiliary device path for ncu: receptor
    grids on the device (N=128 bench pair), the LSE adjoint with ligand-grid
    gradients, pose scores and the detail score terms (N=96, 150/70 pair)."""
    import numpy as np
    import torch

    from megadock_b200 import FFTProcess, Job, POSE_DTYPE, rotation_matrices, synth
    with tempfile.TemporaryDirectory() as tmp:
        rp, lp = make_inputs(tmp)
        job = Job(["-R", rp, "-L", lp, "-F", str(N_FFT), "-r", "24"])
        fp = FFTProcess(0)
        fp.alloc_array(job.nf1, job.grid_width, job.grid_coord())
        xyz, rad, q, ace = job.receptor_atoms()
        rc, _ = job.centers()
        fp.receptor_build((xyz - np.asarray(rc, np.float32)).astype(np.float32), rad, q, ace)
        fp.fft_memory_free()
        rp, lp = synth.write_pair(tmp, 150, 70, 0, stem="aux")
        job = Job(["-R", rp, "-L", lp, "-F", "96", "-r", "360", "-O", "-N", "200", "-o", os.path.join(tmp, "a.out")])
        fp = FFTProcess(0)
        fp.alloc_array(job.nf1, job.grid_width, job.grid_coord())
        rr, ri = job.receptor_grids()
        fp.receptor_fft(rr, ri)
        x2, r2, q2 = job.ligand_atoms()
        fp.ligand_data_transfer_gpu(x2, r2, q2, job.lig_core)
        fp.set_batch(64)
        mats = rotation_matrices(job.rotation_angles())
        top1 = fp.cuda_fft(mats, t=1).copy()
        fp.adjoint_lse(mats, top1, 10.0, 1.0, lig_rot=[int(np.argmax(top1["score"]))])
        fp.pose_scores(mats[:64], top1[:64])
        job.run(fp)                       # -O: the detail score terms
        torch.cuda.synchronize()
        fp.fft_memory_free()
    print("profile aux done")


def run_pairs_workload(args):
    """64 synthetic pairs, chain lengths log-uniform in 60-800 residues, each
    docked over 3,600 rotations (t=1) in one captured graph: rotation
    evaluations per second summed over pairs (pair-evaluations/s)."""
    import collections

    import torch

    from megadock_b200.pairs import uneven_workload
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    pb = uneven_workload(npairs=64, rotation_set=3600, t=1, stream=stream.cuda_stream)
    for _ in range(args.warmup):
        pb.run()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with Clocks(0) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            pb.run()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    evals = len(pb.ctxs) * pb.n_rot
    sizes = collections.Counter(pb.sizes())
    line = {
        "metric": "pair-evaluations/sec, 64 uneven pairs, 3,600 rotations each (batched form)",
        "value": evals / (ms * 1e-3), "unit": "rotation-evaluations/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "64 synthetic pairs, chains log-uniform 60-800 residues, t=1",
                   "fft_sizes": {str(k): v for k, v in sorted(sizes.items())},
                   "rotations_per_launch": {str(k): v for k, v in sorted(pb.batch_by_n.items())},
                   "inverse_plane_plan": {str(k): v for k, v in sorted(pb.plan_by_n.items())},
                   "xline_tile": {str(k): v for k, v in sorted(pb.tile_by_n.items())}},
        "pairs_per_s": len(pb.ctxs) / (ms * 1e-3),
        "clocks": clk.summary(),
    }
    print(json.dumps(line, default=float))


def _timed_wall(fn, steps, warmup):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        fn()
    torch.cuda.synchronize()
    return 1000.0 * (time.perf_counter() - t0) / steps


def run_adjoint_workload(args):
    """The 150/70-residue pair at N = 96, 3,600 rotations: one step = the
    batched forward (t = 1, device-resident rotations and poses) plus the
    adjoint of T * log(sum_r exp(s_r / T)) at T = 10 through the C ABI (top-1
    poses in, receptor / charge / alpha gradients out)."""
    import numpy as np
    import torch

    from megadock_b200 import FFTProcess, Job, POSE_DTYPE, rotation_matrices, synth
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    with tempfile.TemporaryDirectory() as tmp:
        rp, lp = synth.write_pair(tmp, 150, 70, 0, stem="adj")
        job = Job(["-R", rp, "-L", lp, "-F", "96", "-r", "3600"])
        rr, ri = job.receptor_grids()
        xyz, rad, q = job.ligand_atoms()
    mats = rotation_matrices(job.rotation_angles())
    n = len(mats)
    fp = FFTProcess(0, stream=stream.cuda_stream)
    fp.alloc_array(job.nf1, job.grid_width, job.grid_coord())
    fp.receptor_fft(rr, ri)
    fp.ligand_data_transfer_gpu(xyz, rad, q, job.lig_core)
    d_rot = torch.from_numpy(mats).cuda()
    d_pose = torch.zeros(n * 5, dtype=torch.int32, device="cuda")
    if args.batch:
        fp.set_batch(args.batch)
    else:
        from megadock_b200.tune import autotune
        autotune(fp, d_rot.data_ptr(), d_pose.data_ptr(), 1)
    state = {}

    def fwd():
        fp.dock_device(d_rot.data_ptr(), 0, n, 1, d_pose.data_ptr())

    def step():
        fwd()
        top1 = d_pose.cpu().numpy().view(POSE_DTYPE)
        state["res"] = fp.adjoint_lse(mats, top1, 10.0, 1.0)
        state["live"] = int((top1["score"] > 0).sum())

    with Clocks(0) as clk:
        ms = _timed_wall(step, args.steps, args.warmup)
    ms_fwd = _timed_wall(fwd, args.steps, 1)
    top1 = d_pose.cpu().numpy().view(POSE_DTYPE)
    s = top1["score"].astype(np.float64)
    w = np.exp((s - s.max()) / 10.0)
    w /= w.sum()
    nz = int((w.astype(np.float32) != 0).sum())
    line = {
        "metric": "rotations/sec, forward + adjoint of LSE(T=10) over per-rotation top-1 scores, 96^3, 3,600 rot",
        "value": n / (ms * 1e-3), "unit": "rotations/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"adjoint, 150/70-residue synthetic pair ({job.na_rec}/{job.na_lig} atoms), N=96, "
                               f"3600 rotations, t=1, T=10", "timing": "wall clock around synchronous C-ABI calls"},
        "forward_ms": ms_fwd, "adjoint_ms": ms - ms_fwd, "rotations_with_weight": nz,
        "loss": state["res"]["loss"], "d_alpha": state["res"]["d_alpha"],
        "clocks": clk.summary(),
    }
    fp.fft_memory_free()
    print(json.dumps(line, default=float))


def run_fit_workload(args):
    """32 planted complexes (chains log-uniform in 200-1,500 residues), the
    54,000-rotation set, N chosen per pair: one step = the forward (batched,
    t = 1) and the ranking-loss adjoint of every pair at the current alpha and
    charge scales, i.e. one gradient evaluation of the fit."""
    import collections

    import torch

    from megadock_b200 import synth
    from megadock_b200.fit import Fitter, FitPair
    from megadock_b200.pairs import choose_fft_size
    torch.cuda.set_device(0)
    t_setup = time.perf_counter()
    tmp = tempfile.mkdtemp(prefix="md_fit_")
    pairs = []
    for nr, nl, seed in synth.fitting_pairs(args.fit_pairs):
        pc = synth.plant_complex(tmp, nr, nl, seed, rotation_set=54000)
        pairs.append(FitPair(pc, choose_fft_size(pc.rec_pdb, pc.lig_pdb), 54000, batch=args.batch or None,
                             tune=not args.batch))
    t_setup = time.perf_counter() - t_setup
    f = Fitter(pairs, alpha=1.0, temperature=10.0)
    state = {}

    def step():
        state["eval"] = f.evaluate()

    with Clocks(0) as clk:
        ms = _timed_wall(step, args.steps, args.warmup)
    loss, ga, gs, stats = state["eval"]
    evals = sum(len(p.mats) for p in pairs)
    sizes = collections.Counter(p.N for p in pairs)
    line = {
        "metric": "pair-evaluations/sec, forward + ranking-loss adjoint, 32 planted pairs, 54,000 rotations each",
        "value": evals / (ms * 1e-3), "unit": "rotation-evaluations/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{len(pairs)} planted complexes, chains log-uniform 200-1500 residues, "
                               "54000 rotations, t=1, T=10, negatives > 10 A C-alpha RMSD",
                   "fft_sizes": {str(k): v for k, v in sorted(sizes.items())},
                   "timing": "wall clock around synchronous C-ABI calls, host label and chain-rule work included"},
        "loss": loss, "d_alpha": ga, "adjoint_poses": int(sum(st["n_adj"] for st in stats)),
        "positive_rank_median": float(statistics.median(st["rank"] for st in stats)),
        "setup_s": t_setup, "clocks": clk.summary(),
    }
    print(json.dumps(line, default=float))


def cufft_comparator(fp, job, mats, rr, ri, d_pose, stream, steps, warmup, batch=16):
    """The same workload's score grids through the CUDA FFT library (torch.fft):
    forward C2C, conj(R^) product, inverse C2C and top-t, timed with CUDA
    events over `batch` rotations whose ligand grids (the library's voxelizer)
    are already resident; their top scores are checked against the fused
    pipeline's records of the same rotations."""
    import numpy as np
    import torch

    from megadock_b200 import cufft_check as CF
    vox = [fp.ligand_voxels(m) for m in mats[:batch]]
    lig = CF.embed(np.stack([v[0] for v in vox]), np.stack([v[1] for v in vox]), job.nf1)
    rhat = CF.receptor_spectrum(rr, ri, job.nf1)

    def step():
        sg = CF.scores(rhat, lig)
        return torch.topk(sg.reshape(batch, -1), T_POSES, dim=1)

    for _ in range(max(warmup, 3)):
        step()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    want = CF.top_t(CF.scores(rhat, lig), T_POSES)[0]
    got = d_pose[:batch * T_POSES * 5].view(torch.float32).reshape(batch, T_POSES, 5)[..., 0].cpu().numpy()
    rel = float(np.max(np.abs(got - want) / np.maximum(np.abs(want), 1e-30)))
    return {"value": batch / (ms * 1e-3), "unit": "rotations/s", "ms_per_launch": ms, "rotations_per_launch": batch,
            "what": "torch.fft (CUDA FFT library) C2C forward + conj(R^) product + C2C inverse + top-t per "
                    "rotation; ligand grids precomputed and resident, so voxelization is not timed",
            "max_rel_diff_top_scores_vs_fused": rel}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=0, help="rotations per launch (0 = autotune batch and plan)")
    ap.add_argument("--plan", type=int, default=0,
                    help="inverse plane kernel radix plan with --batch or --profile-case (0, 1, 2)")
    ap.add_argument("--tile", type=int, default=32,
                    help="x-line kernel kz lines per CTA with --batch or --profile-case (8, 16, 32)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-cufft", action="store_true", help="skip the cuFFT comparator leg")
    ap.add_argument("--workload", default="metric", choices=["metric", "pairs", "adjoint", "fit"],
                    help="metric: the headline workload; pairs: 64 uneven synthetic pairs, 3,600 rotations each; "
                         "adjoint: forward + LSE adjoint at 96^3, 3,600 rotations; fit: one ranking-loss gradient "
                         "evaluation over 32 planted pairs, 54,000 rotations each")
    ap.add_argument("--fit-pairs", type=int, default=32)
    ap.add_argument("--fft", type=int, default=0, metavar="N",
                    help="FFT edge of --profile-case (default 128; the bench pair fits every built size)")
    ap.add_argument("--profile-case", type=int, default=0, metavar="R",
                    help="run R rotations of the batched form once (for ncu captures) and exit")
    ap.add_argument("--profile-aux", action="store_true",
                    help="one small run of the receptor-grid, adjoint, pose-score and detail kernels (for ncu)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.profile_case:
        return run_profile_case(args)
    if args.profile_aux:
        return run_profile_aux(args)
    if args.workload == "pairs":
        return run_pairs_workload(args)
    if args.workload == "adjoint":
        return run_adjoint_workload(args)
    if args.workload == "fit":
        return run_fit_workload(args)

    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one rank per GPU: run this same command under torch.distributed.run
        import socket

        from megadock_b200.shard import torchrun_command
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        cmd = torchrun_command(str(Path(__file__).resolve()), sys.argv[1:], args.gpus, port)
        raise SystemExit(subprocess.run(["timeout", "-k", "60", "1800", *cmd]).returncode)
    return run_metric(args)


def parity_vs_golden(poses):
    """Check the records of the timed run (n_rot x t poses, rotation order)
    against the reference's per-rotation top-3 of every 15th rotation
    (tests/golden/bench_n128_D_t3_rot.npz, written by the reference's own CPU
    code): largest relative score difference against its FP32 and FP64 FFT
    paths and the number of equal cells."""
    import numpy as np
    path = ROOT / "tests" / "golden" / "bench_n128_D_t3_rot.npz"
    if not path.exists():
        return {"error": f"{path.name} missing"}
    g = np.load(path)
    rots = g["rot"]
    rec = poses.reshape(-1, T_POSES)[rots]
    score = rec["score"].astype(np.float64)
    cell = np.stack([rec["i"], rec["j"], rec["k"]], -1)
    rel32 = np.abs(score - g["score32"]) / np.abs(g["score32"])
    rel64 = np.abs(score - g["score64"]) / np.abs(g["score64"])
    ok_rot = bool((rec["rot"] == rots[:, None]).all())
    return {"rotations_checked": int(len(rots)), "poses_checked": int(rec.size),
            "max_rel_vs_reference_fp32": float(rel32.max()), "max_rel_vs_fp64": float(rel64.max()),
            "within_1e-4": bool((rel32 <= 1e-4).all() and (rel64 <= 1e-4).all()),
            "cells_equal": int((cell == g["cell32"]).all(-1).sum()), "rotation_indices_ok": ok_rot,
            "source": "every 15th rotation of the 54,000 set, reference CPU code (FP32 FFT and FP64 FFT)"}


def run_metric(args):
    import numpy as np
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    # collectives over NCCL, one GPU per rank; MD_BENCH_BACKEND=gloo runs them
    # on host copies and lets ranks share GPUs (tests on a one-GPU machine)
    backend = os.environ.get("MD_BENCH_BACKEND", "nccl")
    gpu = local if backend == "nccl" else local % max(torch.cuda.device_count(), 1)
    torch.cuda.set_device(gpu)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        if backend == "nccl":
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device(f"cuda:{gpu}"))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    coll = f"cuda:{gpu}" if backend == "nccl" else "cpu"   # where collective tensors live

    from megadock_b200 import POSE_DTYPE, FFTProcess, Job, rotation_matrices
    from megadock_b200.shard import gather_records, max_over_ranks, shard_range
    from megadock_b200.tune import autotune

    # a dedicated stream: the library captures CUDA graphs on it, which the
    # legacy default stream does not allow
    stream = torch.cuda.Stream(device=gpu)
    torch.cuda.set_stream(stream)
    dev = f"cuda:{gpu}"
    with tempfile.TemporaryDirectory() as tmp:
        rp, lp = make_inputs(tmp)
        config = workload_config(rp, lp)
        job = Job(["-R", rp, "-L", lp, "-F", str(N_FFT), "-t", str(T_POSES), "-D", "-o",
                   os.path.join(tmp, "bench.out")])
        rr, ri = job.receptor_grids()
        xyz, rad, q = job.ligand_atoms()
        mats = rotation_matrices(job.rotation_angles())
        nrot = len(mats)
        # this rank's block of the one job (the whole job at one GPU)
        r0, r1 = shard_range(nrot, rank, world)
        nloc = r1 - r0
        fp = FFTProcess(gpu, stream=stream.cuda_stream)
        fp.alloc_array(job.nf1, job.grid_width, job.grid_coord())
        fp.receptor_fft(rr, ri)
        fp.ligand_data_transfer_gpu(xyz, rad, q, job.lig_core)
        d_rot = torch.from_numpy(np.ascontiguousarray(mats[r0:r1])).to(dev)
        d_pose = torch.zeros(nloc * T_POSES * 5, dtype=torch.int32, device=dev)

        if args.batch:
            batch, plan = args.batch, args.plan
            fp.set_plan(plan)
            fp.set_tile(args.tile)
        else:
            batch, plan = autotune(fp, d_rot.data_ptr(), d_pose.data_ptr(), T_POSES)
        tile = fp.tile
        merged = {}

        def timed(fn, steps, warmup):
            for _ in range(warmup):
                fn()
            torch.cuda.synchronize()
            if dist:
                dist.barrier()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            if dist:
                ms = max_over_ranks(ms, device=coll)
                dist.barrier()
            return ms / steps

        def dev_step():
            fp.dock_device(d_rot.data_ptr(), r0, nloc, T_POSES, d_pose.data_ptr())
            if dist:
                # the job's exchange step: every rank's records, in rotation order
                merged["all"] = gather_records(d_pose if coll != "cpu" else d_pose.cpu(), nrot, T_POSES)

        # batched, device-resident inputs
        fp.set_batch(batch)
        with Clocks(gpu) as clk:
            ms_batched = timed(dev_step, args.steps, args.warmup)
        all_rec = merged["all"] if dist else d_pose
        poses_timed = all_rec.cpu().numpy().view(POSE_DTYPE).copy() if rank == 0 else None
        # plain form (one rotation per pipeline, no graph): its per-rotation
        # cost does not depend on the rotation count, so it is timed on the
        # first PLAIN_SAMPLE rotations of this rank's block
        fp.set_batch(1)
        ns = min(PLAIN_SAMPLE, nloc)

        def plain_step():
            fp.dock_device(d_rot.data_ptr(), r0, ns, T_POSES, d_pose.data_ptr())

        ms_plain = timed(plain_step, args.steps, 1) * nloc / ns
        # e2e through the C ABI with host buffers: receptor grids, ligand and
        # this block's rotation matrices in, poses out; rank 0 gathers the
        # records (host gather)
        fp.set_batch(batch)
        host_rot = np.ascontiguousarray(mats[r0:r1])

        def e2e_step():
            fp.receptor_fft(rr, ri)
            fp.ligand_data_transfer_gpu(xyz, rad, q, job.lig_core)
            out = fp.cuda_fft(host_rot, t=T_POSES, first_rot=r0)
            if dist:
                from megadock_b200.shard import gather_poses
                gather_poses(out)

        for _ in range(args.warmup):
            e2e_step()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        torch.cuda.synchronize()
        ms_e2e = 1000.0 * (time.perf_counter() - t0) / args.steps
        if dist:
            ms_e2e = max_over_ranks(ms_e2e, device=coll)
        # per-stage profile of the batched form (events on the launch stream)
        stage_ms, launches_prof = fp.dock_profile(d_rot.data_ptr(), r0, nloc, T_POSES, d_pose.data_ptr())
        launches_all = launches_prof
        if dist:
            t_l = torch.tensor([launches_prof], dtype=torch.int64, device=coll)
            dist.all_reduce(t_l)
            launches_all = int(t_l.item())
        cufft = None
        if rank == 0 and not args.no_cufft:
            try:
                cufft = cufft_comparator(fp, job, mats[r0:r1], rr, ri, d_pose, stream, args.steps, args.warmup)
            except Exception as e:  # a comparator, never required
                cufft = {"error": str(e)[:200]}
        fp.fft_memory_free()

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return

    N3 = N_FFT ** 3
    nb_launches = -(-nloc // batch)
    # algorithmic DRAM bytes per rotation per stage (complex64 = 8 B, NG = N/2)
    NG = N_FFT // 2
    stage_bytes = {
        "voxelize": NG ** 3 // 4,                    # two class bit planes per voxel plane
        "plane_fwd": NG ** 3 // 4 + 4 * N3,           # read them, write ng spectrum planes (N^2 each)
        "xline": 4 * N3 + 4 * N3,                     # read those, write the Hermitian half (N/2 rows)
        "plane_inv": 4 * N3,                          # read the half once
        "merge": 0,
    }
    names = ["voxelize", "plane_fwd", "xline", "plane_inv", "merge"]
    dom = max(range(5), key=lambda k: stage_ms[k])
    # R^ is read once per launch (it is shared by the launch's rotations)
    dom_bytes_launch = stage_bytes[names[dom]] * batch + (8 * N3 if names[dom] == "xline" else 0)
    dom_ms_launch = stage_ms[dom] / nb_launches
    peak, peak_kind = _peaks()
    achieved = dom_bytes_launch / (dom_ms_launch * 1e-3) / 1e9
    # DRAM bytes per rotation per stage from one ncu capture of this pipeline
    # at N=128, 64 rotations per launch (dram__bytes_read.sum +
    # dram__bytes_write.sum per launch / 64, profiles/ncu_dock_kernels_n128_b64.md);
    # scaled by rotations per launch (R^, read once per launch by xline, adds
    # 16.8 MB per launch and is left in the xline figure)
    traffic_per_rotation = {"voxelize": 79.4e3, "plane_fwd": 7.54e6, "xline": 17.08e6, "plane_inv": 8.45e6,
                            "merge": 3.3e3}
    traffic = traffic_per_rotation[names[dom]] * batch if N_FFT == 128 else None
    value = nrot / (ms_batched * 1e-3)
    plain = nrot / (ms_plain * 1e-3)
    e2e = nrot / (ms_e2e * 1e-3)
    model_bytes = 52 * N3
    pipe_bytes = sum(stage_bytes.values())
    line = {
        "metric": METRIC, "value": value, "unit": "rotations/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_batched, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {**config, "rotations_per_launch": batch,
                   "inverse_plane_plan": plan, "xline_tile": tile, "groups_in_flight": fp.lanes,
                   "l2": "working set per step >> L2 (54,000 rotations x ~25 MB of intermediates)",
                   "parallelism": f"rotation shards x{world}" + (", NCCL all-gather of the records" if dist else "")},
        "plain": {"value": plain, "ms_per_step": ms_plain, "unit": "rotations/s",
                  "sample": f"first {ns} rotations of each rank's block per step, scaled to the block"},
        "batched_over_plain": value / plain,
        "e2e": {"value": e2e, "unit": "rotations/s", "ms_per_step": ms_e2e,
                "h2d_bytes_per_step": int(world * (rr.nbytes + ri.nbytes + xyz.nbytes + rad.nbytes + q.nbytes)
                                          + mats.nbytes),
                "d2h_bytes_per_step": int(nrot * T_POSES * 20)},
        "roofline": {"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "stage_ms": {n: float(stage_ms[k]) for k, n in enumerate(names)}},
        "pipeline_bytes_per_rotation": {"model_52N3": model_bytes, "this_pipeline": pipe_bytes},
        "pipeline_model": {"bytes_per_rotation": model_bytes,
                           "achieved_GBps": model_bytes * value / 1e9,
                           "frac": model_bytes * value / 1e9 / (peak * world)},
        "pipeline_own_bytes": {"bytes_per_rotation": pipe_bytes, "achieved_GBps": pipe_bytes * value / 1e9,
                               "frac": pipe_bytes * value / 1e9 / (peak * world)},
        "parity": parity_vs_golden(poses_timed),
        "gpu_launches": int(args.steps * launches_all),
        "clocks": clk.summary(),
    }
    if cufft is not None:
        line["cufft_comparator"] = cufft
    if not args.no_cpu_baseline:
        try:
            from oracle import ref
            if ref.available():
                with tempfile.TemporaryDirectory() as tmp:
                    rp2, lp2 = make_inputs(tmp)
                    v, cores, secs = cpu_reference(rp2, lp2)
                line["cpu_baseline"] = {"value": v, "unit": "rotations/s", "cores": cores, "kind": "reference",
                                        "fft": "project-written scalar FFTW-API shim (libfftw3f is not on the image)",
                                        "sample": f"{REF_SAMPLE_ROT} rotations of the same job ({secs:.1f} s)"}
                with tempfile.TemporaryDirectory() as tmp:
                    rp2, lp2 = make_inputs(tmp)
                    line["cpu_baseline"]["production_fft"] = cpu_production_fft(rp2, lp2)
        except Exception as e:  # the baseline is reported, never required
            line["cpu_baseline"] = {"error": str(e)[:200]}
    print(json.dumps(line, default=float))
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
