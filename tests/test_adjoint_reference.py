"""The FP64 adjoint reference (oracle/adjoint.py) on the CPU: its analytic
gradient of the log-sum-exp loss agrees with its own central finite
differences, and the charge-cell rule it uses reproduces the oracle's charge
grids bit for bit.  The device adjoint is checked against both in
test_gpu_adjoint.py."""
import numpy as np
import pytest


def _problem(pairs, n_rot=48):
    from megadock_b200 import Job, rotation_matrix
    from oracle import adjoint as A
    rp, lp = pairs["small"]
    job = Job(["-R", rp, "-L", lp, "-F", "64", "-r", "360"])
    xyz, rad, q = job.ligand_atoms()
    rr, ri = job.receptor_grids()
    ref = A.AdjointReference(rr, ri, xyz, rad, q, job.grid_width, job.grid_coord(), job.lig_core, job.nf1)
    rots = np.array([rotation_matrix(a) for a in job.rotation_angles()[:n_rot]])
    shifts = np.zeros((n_rot, 3), np.int64)
    scores = np.zeros(n_rot)
    for r in range(n_rot):
        _, gr, gi = ref.ligand(rots[r])
        S, _, _ = ref.fft.scores(gr, gi)
        S = S.reshape(-1)
        am = int(np.argmax(S))
        shifts[r] = (am // job.nf1 ** 2, (am // job.nf1) % job.nf1, am % job.nf1)
        scores[r] = max(S[am], 0.0)
    return job, ref, rots, shifts, scores


@pytest.mark.parametrize("temperature", [10.0, 300.0])
def test_reference_gradient_vs_finite_differences(built, pairs, temperature):
    from oracle import adjoint as A
    job, ref, rots, shifts, scores = _problem(pairs)
    alpha = 1.0
    _, w = A.weights(scores, temperature)
    top = np.argsort(-w)[:3]
    g = ref.run(rots, shifts, scores, temperature, alpha, lig_rot=top, check_cells=True)
    rng = np.random.default_rng(1)
    rec = [(0, x) for x in rng.choice(np.flatnonzero(g["d_rec_r"]), 20, replace=False)]
    rec += [(1, x) for x in rng.choice(np.flatnonzero(g["d_rec_i"]), 20, replace=False)]
    atoms = rng.choice(len(ref.charge), 20, replace=False)
    lig = [(r, p, y) for r in top for p in (0, 1)
           for y in rng.choice(np.flatnonzero(g["d_lig"][r][p]), 5, replace=False)]
    coords = A.Coordinates(rec, atoms, lig, alpha=True)
    out = ref.run(rots, shifts, scores, temperature, alpha, lig_rot=top, coords=coords, check_cells=False)
    assert (out["fd"].arg == shifts).all()
    fd, ok = out["fd"].gradient(np.ones(len(rots), bool), 1e-3, temperature)
    an = np.concatenate([
        [(g["d_rec_r"] if p == 0 else g["d_rec_i"]).reshape(-1)[x] for p, x in rec],
        g["d_charge"][atoms],
        [g["d_lig"][r][p].reshape(-1)[y] for r, p, y in lig],
        [g["d_alpha"]]])
    assert ok.mean() > 0.9
    err = np.abs(an - fd)[ok]
    assert (err <= 1e-6 * np.abs(fd[ok]) + 1e-9 * np.abs(fd).max()).all(), err.max()


def test_shift_index_matches_roll():
    from oracle import adjoint as A
    rng = np.random.default_rng(3)
    ng, N = 6, 12
    g = rng.standard_normal((ng,) * 3)
    emb = np.zeros((N,) * 3)
    emb[3:9, 3:9, 3:9] = g
    for t in [(0, 0, 0), (1, 11, 5), (6, 6, 6), (11, 0, 3)]:
        want = np.roll(emb, [-d for d in t], axis=(0, 1, 2))[3:9, 3:9, 3:9]
        assert np.array_equal(A.shifted(g, N, t), want)


def test_weights_clamped_rotations():
    from oracle import adjoint as A
    loss, w = A.weights([0.0, 10.0, 20.0], 10.0)
    assert w[0] == 0.0 and w[2] > w[1] > 0
    assert np.isclose(loss, 20 + 10 * np.log(np.exp(-2) + np.exp(-1) + 1))


def test_directions_and_fixed_entries(built, pairs):
    """Directions reproduce the single-coordinate differences (alpha as the
    receptor direction Ri / alpha, a charge as a unit atom vector), and a
    ranking loss over a fixed-translation entry plus maxima matches its
    analytic gradient through dl_ds."""
    from oracle import adjoint as A
    job, ref, rots, shifts, scores = _problem(pairs, n_rot=24)
    T, alpha = 10.0, 1.0
    a0 = 3
    unit = np.zeros(len(ref.charge))
    unit[a0] = 1.0
    dirs = [dict(rec_i=ref.rec_i / alpha), dict(atoms=unit),
            dict(rec_r=np.ones_like(ref.rec_r), rec_i=ref.rec_i, atoms=ref.charge.astype(np.float64))]
    # entry 0: rotation 5 at a translation one cell away from its maximiser, held fixed
    rots2 = np.concatenate([rots[5:6], rots])
    sh2 = np.concatenate([(shifts[5:6] + [0, 0, 1]) % job.nf1, shifts])
    fixed = np.zeros(len(rots2), bool)
    fixed[0] = True
    coords = A.Coordinates(atoms=[a0], alpha=True, dirs=dirs)
    out0 = ref.run(rots2, sh2, np.concatenate([[1.0], scores]), T, alpha, coords=coords, fixed=fixed,
                   dl_ds=np.zeros(len(rots2)), check_cells=False)
    fdt = out0["fd"]
    s = fdt.S[fdt.starts]
    s = np.where(fixed, s, np.maximum(s, 0))
    m = s.max()
    p = np.exp((s - m) / T)
    p /= p.sum()
    w = p.copy()
    w[0] -= 1.0
    w[~fixed & (s <= 0)] = 0.0
    loss_fn = lambda v: -v[0] + A._lse(v, T)
    g = ref.run(rots2, sh2, s, T, alpha, dl_ds=w, fixed=fixed, check_cells=False)
    fd, ok = fdt.gradient(np.ones(len(rots2), bool), 1e-3, T, loss_fn=loss_fn)
    assert ok.all()
    # rows: atom a0, dir alpha, dir unit atom, dir mixed, alpha
    an_atom = g["d_charge"][a0]
    an_alpha = g["d_alpha"]
    an_mixed = g["d_rec_r"].sum() + (g["d_rec_i"] * ref.rec_i).sum() + g["d_charge"] @ ref.charge
    want = np.array([an_atom, an_alpha, an_atom, an_mixed, an_alpha])
    assert np.allclose(fd, want, rtol=1e-6, atol=1e-9 * np.abs(want).max()), (fd, want)
