"""Fitting alpha and per-residue charge scales on decoys the docking path
generates (GPU).

  * planted complexes: the native pose (set rotation + grid translation)
    restores the planted ligand (C-alpha RMSD ~0); the best-scoring docking
    pose puts the ligand against the receptor without overlap;
  * md_pose_scores at the per-rotation top-1 poses equals the docking scores;
  * the ranking-loss gradient (device adjoint + chain rule to alpha and the
    charge scales) against the FP64 reference gradient at the same poses and
    weights, and against FP64 central finite differences (step 1e-3) of the
    ranking loss along alpha and three charge-scale directions;
  * a few Adam steps lower the ranking loss.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

T = 10.0


@pytest.fixture(scope="module")
def planted(tmp_path_factory):
    from megadock_b200 import synth
    d = tmp_path_factory.mktemp("planted")
    return [synth.plant_complex(str(d), nr, nl, seed, rotation_set=360)
            for nr, nl, seed in [(70, 30, 4100), (100, 45, 4101)]]


def _pair(pc, rotation_set=360):
    from megadock_b200.fit import FitPair
    from megadock_b200.pairs import choose_fft_size
    return FitPair(pc, choose_fft_size(pc.rec_pdb, pc.lig_pdb), rotation_set, batch=32)


@pytest.fixture(scope="module")
def fit_pairs(built, gpu, planted):
    return [_pair(pc) for pc in planted]


def test_native_pose_and_decoy_geometry(fit_pairs):
    from scipy.spatial import cKDTree
    for p in fit_pairs:
        assert p.native_rmsd_check() < 1e-3
        p.set_params(1.0, np.ones(p.K))
        top1, s_pos = p.forward()
        best = top1[np.argmax(top1["score"])]
        rec_xyz = p.job.receptor_atoms()[0]
        xyz_c = p.xyz.reshape(-1, 3).astype(np.float64)
        t = np.array([best["i"], best["j"], best["k"]], np.int64)
        t = np.where(t >= p.N // 2, t - p.N, t)
        m = p.mats[best["rot"]].astype(np.float64).reshape(3, 3)
        placed = xyz_c @ m.T - t * p.job.grid_width + p.rec_c
        d, _ = cKDTree(rec_xyz.reshape(-1, 3)).query(placed)
        assert 1.5 < d.min() < 6.0, d.min()


def test_pose_scores_match_docking(fit_pairs):
    p = fit_pairs[0]
    p.set_params(1.0, np.ones(p.K))
    top1, _ = p.forward()
    live = top1[top1["score"] > 0]
    s = p.fp.pose_scores(p.mats[live["rot"]], live)
    ref = live["score"].astype(np.float64)
    assert np.all(np.abs(s - ref) <= 1e-4 * np.abs(ref) + 1e-3)


def test_ranking_gradient_vs_fp64(fit_pairs):
    from oracle import adjoint as A
    p = fit_pairs[1]
    rng = np.random.default_rng(7)
    alpha = 0.8
    scale = 1.0 + 0.2 * rng.standard_normal(p.K)
    p.set_params(alpha, scale)
    loss, d_alpha, d_scale, st = p.loss_grad(alpha, scale, T)
    ent, w = st["entries"], st["dl_ds"]
    # the same grids and charges the device used
    U = p.U.astype(np.float64)
    ri = (alpha * (scale @ U)).astype(np.float32).reshape(p.rec_r.shape)
    q = (scale[p.lig_codes] * p.q0).astype(np.float32)
    ref = A.AdjointReference(p.rec_r, ri, p.xyz, p.rad, q, p.job.grid_width, p.job.grid_coord(), p.job.lig_core,
                             p.N, fft=A.TorchFFT("cuda:0"))
    shifts = np.stack([ent["i"], ent["j"], ent["k"]], -1).astype(np.int64)
    fixed = np.zeros(len(ent), bool)
    fixed[0] = True
    types = np.argsort(-np.bincount(p.rec_codes, minlength=p.K))[:3]
    ng3 = p.rec_r.size
    dirs = [dict(rec_i=(scale @ U).reshape(p.rec_r.shape))]
    for k in types:
        dirs.append(dict(rec_i=alpha * U[k].reshape(p.rec_r.shape),
                         atoms=np.where(p.lig_codes == k, p.q0, 0.0).astype(np.float64)))
    coords = A.Coordinates(dirs=dirs)
    out = ref.run(p.mats[ent["rot"]], shifts, ent["score"], T, alpha, coords=coords, dl_ds=w, fixed=fixed)
    # FP64 reference gradient through the same chain rule
    dri = out["d_rec_i"].reshape(-1)
    ref_alpha = dri @ (scale @ U)
    ref_scale = alpha * (U @ dri) + np.bincount(p.lig_codes, weights=p.q0 * out["d_charge"], minlength=p.K)
    print(f"\nranking gradient: d_alpha device {d_alpha:.6g} FP64 {ref_alpha:.6g}; "
          f"max |d_scale diff| {np.abs(d_scale - ref_scale).max():.3g} of {np.abs(ref_scale).max():.3g}")
    assert abs(d_alpha - ref_alpha) <= 1e-5 * abs(ref_alpha)
    assert np.abs(d_scale - ref_scale).max() <= 1e-5 * np.abs(ref_scale).max()
    # FP64 central differences of the ranking loss
    fdt = out["fd"]
    keep = fixed | (fdt.arg == shifts).all(1) | (ent["score"] <= 0)
    assert keep.all(), int((~keep).sum())
    fd, ok = fdt.gradient(np.ones(len(ent), bool), 1e-3, T, loss_fn=lambda v: -v[0] + A._lse(v, T))
    an = np.concatenate([[d_alpha], d_scale[types]])
    rel = np.abs(an - fd) / np.abs(fd)
    print(f"ranking loss vs FP64 finite differences: {ok.sum()} of {len(ok)} directions, "
          f"max relative error {rel[ok].max():.3g}")
    assert ok.all() and rel.max() <= 1e-3, (an, fd)


def test_fit_lowers_ranking_loss(fit_pairs):
    from megadock_b200.fit import Fitter
    f = Fitter(fit_pairs, alpha=1.0, temperature=T, lr=0.05)
    first, _ = f.step()
    for _ in range(7):
        last, stats = f.step()
    final, _, _, _ = f.evaluate()
    print(f"\nfit: loss {first:.4g} -> {final:.4g}, alpha {f.alpha:.4g}")
    assert final < first
