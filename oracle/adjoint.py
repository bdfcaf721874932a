"""FP64 reference for the adjoint of the log-sum-exp loss over per-rotation
top-1 scores.  TEST INFRASTRUCTURE: only tests may import this module; it
checks md_adjoint_lse and is never part of the product path.

MEGADOCK itself does not differentiate its scores; the scoring function
whose gradient this restates is the reference's per-rotation score grid

    S_r(t) = Re sum_x conj(R(x)) L_r(x + t)
           = sum_x Rr(x) Lr_r(x + t) + Ri(x) Li_r(x + t)

(complex receptor grid R = Rr + i Ri, src/receptor.cpp; ligand grid of
rotation r, src/ligand.cpp; product with the conjugated receptor spectrum and
inverse FFT, src/fft_process.cpp:333-346 and :441-446; ng^3 grids embedded at
offset N/4 of the N^3 FFT box, src/fft_process.cpp:306-330), the top-1 score
s_r = max(0, max_t S_r(t)) (src/fft_process.cpp:356-376 keeps a running
maximum that starts at 0) and the loss

    L = T * log(sum_r exp(s_r / T)).

Its gradient collapses to shifted grids at the selected translations t*_r:

    dL/dR(x)    = sum_r w_r L_r(x + t*_r),     w_r = softmax(s_r / T), 0 if s_r = 0
    dL/dL_r(y)  = w_r R(y - t*_r)
    dL/dq_a     = sum_r w_r Ri(c_r(a) - t*_r)  (c_r(a): the atom's charge cell)
    dL/dalpha   = sum_x dL/dRi(x) Ri(x) / alpha   (Ri = alpha * U, support fixed)

Finite differences: S_r is linear in every parameter, so a perturbation by
+-h of one parameter moves S_r(t) by +-h * coef_r(t).  The perturbed maximum
can only be reached at translations within 2 h max|coef| of the top; those
candidate sets, computed once from the FP64 score grids, give the perturbed
losses exactly, and a central difference of step h is checked against the
gradient wherever no rotation's maximising translation changes within +-h.
"""
from __future__ import annotations

import numpy as np

from . import oracle as O


def shift_index(ng: int, N: int, d: int) -> np.ndarray:
    """For voxel a in [0, ng): the voxel at FFT position (a + d) mod N of the
    grid embedded at offset N/4, or -1 where that position is zero padding."""
    off = N // 4
    y = (np.arange(ng) + off + d) % N - off
    y[(y < 0) | (y >= ng)] = -1
    return y


def shifted(grid: np.ndarray, N: int, t) -> np.ndarray:
    """out[x] = grid[x + t] (circular FFT coordinates, zero outside)."""
    ng = grid.shape[0]
    idx = [shift_index(ng, N, int(d)) for d in t]
    g = grid[np.ix_(*[np.maximum(i, 0) for i in idx])]
    m = [(i >= 0) for i in idx]
    return g * (m[0][:, None, None] & m[1][None, :, None] & m[2][None, None, :])


def charge_cells(xyz_rot: np.ndarray, ng: int, grid_width: float) -> np.ndarray:
    """The charge cell of every atom: clamp((int)((c + pad) / gw)) in float32,
    pad = ng * gw / 2 (src/ligand.cpp:219-221)."""
    gw = np.float32(grid_width)
    pad = np.float32(np.float32(ng) * gw) / np.float32(2)
    c = ((np.asarray(xyz_rot, np.float32) + pad) / gw).astype(np.int32)
    return np.clip(c, 0, ng - 1)


def weights(scores, temperature: float):
    """(loss, w) in float64; rotations with score <= 0 carry weight 0."""
    s = np.asarray(scores, np.float64)
    m = s.max()
    e = np.exp((s - m) / temperature)
    z = e.sum()
    w = np.where(s > 0, e / z, 0.0)
    return m + temperature * np.log(z), w


class NumpyFFT:
    """FP64 FFTs on the host.  Grids are ng^3, embedded at offset N/4 of the
    N^3 box; correlate(A, B)(t) = sum_x Re(conj(a(x)) b(x + t)) from the
    spectra A, B of a and b."""

    def spectrum(self, re, im=None):
        z = O.embed(re, np.zeros_like(re) if im is None else im, self.N)
        return np.fft.fftn(z)

    def correlate(self, A, B):
        return np.fft.ifftn(np.conj(A) * B).real

    def grids(self, rec_r, rec_i, N):
        self.N = N
        self.R = self.spectrum(rec_r, rec_i)
        self.Ri = self.spectrum(rec_i)

    def scores(self, lig_r, lig_i):
        """(S, E, L): the score grid (the unnormalised inverse FFT divided by
        N^3), its electrostatic part and the ligand spectrum, float64."""
        L = self.spectrum(lig_r, lig_i)
        return self.correlate(self.R, L), self.correlate(self.Ri, self.spectrum(lig_i)), L


class TorchFFT(NumpyFFT):
    """FP64 FFTs on a CUDA device through torch (a checker only)."""

    def __init__(self, device="cuda:0"):
        import torch
        self.torch = torch
        self.dev = device

    def _embed(self, g):
        torch = self.torch
        N, ng = self.N, g.shape[0]
        off = (N - ng) // 2
        z = torch.zeros((N,) * 3, dtype=torch.float64, device=self.dev)
        z[off:off + ng, off:off + ng, off:off + ng] = torch.from_numpy(np.asarray(g, np.float64)).to(self.dev)
        return z

    def spectrum(self, re, im=None):
        torch = self.torch
        z = self._embed(re) if im is None else torch.complex(self._embed(re), self._embed(im))
        return torch.fft.fftn(z)

    def correlate(self, A, B):
        return self.torch.fft.ifftn(self.torch.conj(A) * B).real


def _gather(G, part, ijk, t, N):
    """G[part, ijk + t] per row (circular FFT coordinates, 0 in the padding)."""
    ng = G.shape[1]
    idx = [shift_index(ng, N, int(t[d]))[ijk[:, d]] for d in range(3)]
    ok = (idx[0] >= 0) & (idx[1] >= 0) & (idx[2] >= 0)
    out = np.zeros(len(ijk))
    out[ok] = G[part[ok], idx[0][ok], idx[1][ok], idx[2][ok]]
    return out


def _to_np(a):
    return a if isinstance(a, np.ndarray) else a.cpu().numpy()


def _take(grid, idx):
    if isinstance(grid, np.ndarray):
        return grid.reshape(-1)[idx]
    import torch
    return grid.reshape(-1)[torch.from_numpy(idx).to(grid.device)].cpu().numpy()


def _candidates(S, E, h, coef_max, alpha):
    """(top, argmax, candidates, S at them, E at them): every translation whose
    score is within 2 h max|coef| of the top, the maximiser (lowest linear
    index among equal maxima) first.  alpha: include the electrostatic
    coefficient E / alpha in the bound (None: no alpha coordinate)."""
    if isinstance(S, np.ndarray):
        Sf, Ef = S.reshape(-1), E.reshape(-1)
        top = float(Sf.max())
        am = int(np.argmax(Sf))
        emax = float(np.abs(Ef).max())
        nz = lambda m: np.nonzero(m)[0]
        take = lambda a, i: a[i]
    else:
        import torch
        Sf, Ef = S.reshape(-1), E.reshape(-1)
        top = float(Sf.max())
        am = int(torch.argmax(Sf))
        emax = float(Ef.abs().max())
        nz = lambda m: torch.nonzero(m).flatten().cpu().numpy()
        take = lambda a, i: a[torch.from_numpy(i).to(a.device)].cpu().numpy()
    maxc = max(coef_max, emax / abs(alpha) if alpha else 0.0)
    cand = nz(Sf >= top - (2.0 * h * maxc * 1.01 + 1e-9))
    cand = np.concatenate([[am], cand[cand != am]]).astype(np.int64)
    return top, am, cand, take(Sf, cand), take(Ef, cand)


def _ijk(flat, N):
    return np.stack([flat // (N * N), (flat // N) % N, flat % N], -1)


class Coordinates:
    """Parameters for the finite-difference check: receptor cells (part 0 real,
    1 imaginary, flat ng^3 index), ligand atoms (charges), ligand cells of
    selected rotations (rotation index, part, flat index) and alpha."""

    def __init__(self, rec=(), atoms=(), lig=(), alpha=False, dirs=()):
        self.rec = [(int(p), int(x)) for p, x in rec]
        self.atoms = [int(a) for a in atoms]
        self.lig = [(int(r), int(p), int(y)) for r, p, y in lig]
        self.alpha = bool(alpha)
        # directions in parameter space: dict(rec_r=grid, rec_i=grid, atoms=vector),
        # any key optional; the coordinate moves the receptor grids by h * rec_*
        # and the ligand charges by h * atoms
        self.dirs = list(dirs)

    def __len__(self):
        return len(self.rec) + len(self.atoms) + len(self.lig) + len(self.dirs) + int(self.alpha)


class AdjointReference:
    """One pass over the rotations: FP64 score grids, the reference gradient at
    given translations and weights, and candidate sets with the coefficient of
    every finite-difference coordinate at every candidate."""

    def __init__(self, rec_r, rec_i, xyz_centred, radius, charge, grid_width, grid_coord, lig_core, N,
                 fft=None):
        self.rec_r = np.asarray(rec_r, np.float32)
        self.rec_i = np.asarray(rec_i, np.float32)
        self.ng = self.rec_r.shape[0]
        self.N = N
        self.xyz = np.asarray(xyz_centred, np.float32)
        self.radius = np.asarray(radius, np.float32)
        self.charge = np.asarray(charge, np.float32)
        self.gw = grid_width
        self.gc = np.asarray(grid_coord, np.float32)
        self.core = lig_core
        self.fft = fft or NumpyFFT()
        self.fft.grids(self.rec_r, self.rec_i, N)
        self.max_rec = float(max(np.abs(self.rec_r).max(), np.abs(self.rec_i).max()))
        self.rec2 = np.stack([self.rec_r, self.rec_i])

    def ligand(self, m9):
        """Rotated coordinates and the ligand grids (oracle restatement)."""
        xr = O.rotate(self.xyz, m9)
        gr, gi = O.ligand_grids(xr, self.radius, self.charge, self.ng, self.gw, self.gc, self.core)
        return xr, gr, gi

    def run(self, rotmats, shifts, scores, temperature, alpha, lig_rot=(), coords: Coordinates | None = None,
            h=1e-3, check_cells=True, dl_ds=None, fixed=None):
        """rotmats (n, 9); shifts (n, 3) and scores (n,) are the translations and
        top-1 scores the gradient is taken at (e.g. the device's).  dl_ds
        replaces the log-sum-exp weights by given ones; fixed[n] marks entries
        whose score is the value at the given translation (not a maximum over
        translations, not clamped at 0).  Returns the reference gradient (dict)
        and, with coords, the finite-difference tables."""
        ng, N = self.ng, self.N
        n = len(rotmats)
        loss, w = weights(scores, temperature)
        if dl_ds is not None:
            loss, w = None, np.asarray(dl_ds, np.float64)
        fixed = np.zeros(n, bool) if fixed is None else np.asarray(fixed, bool)
        dRr = np.zeros((ng,) * 3)
        dRi = np.zeros((ng,) * 3)
        dq = np.zeros(len(self.charge))
        sel = list(lig_rot)
        dL = {r: None for r in sel}
        top64 = np.zeros(n)
        arg64 = np.zeros((n, 3), np.int64)
        cand_S, cand_coef, seg = [], [], [0]
        lig_by_rot = {}
        if coords is not None:
            for k, (r, p, y) in enumerate(coords.lig):
                lig_by_rot.setdefault(r, []).append((k, p, y))
            nrec, nat = len(coords.rec), len(coords.atoms)
            rec_p = np.array([p for p, _ in coords.rec], np.int64).reshape(-1)
            rec_x = np.array([x for _, x in coords.rec], np.int64).reshape(-1)
            rec_ijk = np.stack([rec_x // (ng * ng), (rec_x // ng) % ng, rec_x % ng], -1)
            atoms = np.array(coords.atoms, np.int64)
            nlig = len(coords.lig)
            dir_spec = {}
        for r in range(n):
            xr, gr, gi = self.ligand(rotmats[r])
            cells = charge_cells(xr, ng, self.gw)
            if check_cells:
                acc = np.zeros((ng,) * 3, np.float32)      # float32 sums in atom order (unbuffered add.at)
                np.add.at(acc, (cells[:, 0], cells[:, 1], cells[:, 2]), self.charge)
                if not np.array_equal(acc, gi):
                    raise AssertionError(f"rotation {r}: charge cells do not reproduce the charge grid")
            t = shifts[r]
            if w[r] != 0.0:
                dRr += w[r] * shifted(gr.astype(np.float64), N, t)
                dRi += w[r] * shifted(gi.astype(np.float64), N, t)
                ci = shift_index(ng, N, -int(t[0]))[cells[:, 0]]
                cj = shift_index(ng, N, -int(t[1]))[cells[:, 1]]
                ck = shift_index(ng, N, -int(t[2]))[cells[:, 2]]
                ok = (ci >= 0) & (cj >= 0) & (ck >= 0)
                v = np.zeros(len(cells))
                v[ok] = self.rec_i[ci[ok], cj[ok], ck[ok]]
                dq += w[r] * v
            if r in dL:
                minus = [(-int(d)) for d in t]
                dL[r] = (w[r] * shifted(self.rec_r.astype(np.float64), N, minus),
                         w[r] * shifted(self.rec_i.astype(np.float64), N, minus))
            if coords is None:
                continue
            S, E, Lspec = self.fft.scores(gr, gi)
            lig_max = max(float(np.abs(gr).max()), float(np.abs(gi).max()), self.max_rec)
            dgrids = []
            for k, d in enumerate(coords.dirs):            # dS(t)/d(direction): full grids
                g = None
                if d.get("rec_r") is not None or d.get("rec_i") is not None:
                    if k not in dir_spec:
                        z = np.zeros((ng,) * 3)
                        dir_spec[k] = self.fft.spectrum(d.get("rec_r", z) if d.get("rec_r") is not None else z,
                                                        d.get("rec_i", z) if d.get("rec_i") is not None else z)
                    g = self.fft.correlate(dir_spec[k], Lspec)
                if d.get("atoms") is not None:
                    Q = np.zeros((ng,) * 3)
                    np.add.at(Q, (cells[:, 0], cells[:, 1], cells[:, 2]), np.asarray(d["atoms"], np.float64))
                    ga = self.fft.correlate(self.fft.Ri, self.fft.spectrum(Q))
                    g = ga if g is None else g + ga
                dgrids.append(g)
                lig_max = max(lig_max, float(abs(g).max()))
            if fixed[r]:
                am = int((t[0] * N + t[1]) * N + t[2])
                cand = np.array([am], np.int64)
                Sc = _to_np(S.reshape(-1)[am:am + 1]).astype(np.float64)
                Ec = _to_np(E.reshape(-1)[am:am + 1]).astype(np.float64)
                top = float(Sc[0])
            else:
                top, am, cand, Sc, Ec = _candidates(S, E, h, lig_max, alpha if coords.alpha else None)
            top64[r] = top
            arg64[r] = _ijk(am, N)
            tc = _ijk(cand, N)
            coef = np.zeros((len(coords), len(cand)))
            lig2 = np.stack([gr, gi])
            rows = lig_by_rot.get(r, ())
            for c in range(len(cand)):
                if nrec:                                   # dS(t)/dR(x) = L(x + t)
                    coef[:nrec, c] = _gather(lig2, rec_p, rec_ijk, tc[c], N)
                if nat:                                    # dS(t)/dq_a = Ri(c(a) - t)
                    coef[nrec:nrec + nat, c] = _gather(self.rec2[1:], np.zeros(nat, np.int64), cells[atoms],
                                                       -tc[c], N)
                if rows:                                   # dS_r(t)/dL_r(y) = R(y - t)
                    ks = np.array([k for k, _, _ in rows])
                    ps = np.array([p for _, p, _ in rows], np.int64)
                    ys = np.array([y for _, _, y in rows], np.int64)
                    yijk = np.stack([ys // (ng * ng), (ys // ng) % ng, ys % ng], -1)
                    coef[nrec + nat + ks, c] = _gather(self.rec2, ps, yijk, -tc[c], N)
            for k, g in enumerate(dgrids):
                coef[nrec + nat + nlig + k] = _take(g, cand)
            if coords.alpha:                               # dS(t)/dalpha = E(t) / alpha
                coef[-1] = Ec / alpha
            cand_S.append(Sc)
            cand_coef.append(coef)
            seg.append(seg[-1] + len(cand))
        dalpha = float((dRi * self.rec_i).sum() / alpha) if alpha != 0 else float("nan")
        out = {"loss": loss, "w": w, "d_rec_r": dRr, "d_rec_i": dRi, "d_charge": dq, "d_alpha": dalpha,
               "d_lig": dL}
        if coords is not None:
            out["fd"] = FiniteDifferences(np.concatenate(cand_S), np.concatenate(cand_coef, axis=1),
                                          np.array(seg[:-1]), top64, arg64, ~fixed)
        return out


class FiniteDifferences:
    """Central differences of the FP64 loss from the candidate tables."""

    def __init__(self, S, coef, starts, top, arg, clamp):
        self.S, self.coef, self.starts = S, coef, starts
        self.top, self.arg = top, arg
        self.clamp = clamp

    def _floor(self, s):
        return np.where(self.clamp, np.maximum(s, 0.0), s)

    def losses(self, rot_mask, k, step, temperature, loss_fn=None):
        """(loss, loss with every maximiser held at the unperturbed one) after
        moving coordinate k by step."""
        f = loss_fn or (lambda s: _lse(s, temperature))
        v = self.S + step * self.coef[k]
        s = self._floor(np.maximum.reduceat(v, self.starts))[rot_mask]
        lin = self._floor(v[self.starts])[rot_mask]
        return f(s), f(lin)

    def gradient(self, rot_mask, h, temperature, switch_tol=1e-4, loss_fn=None):
        """(fd, differentiable): per coordinate the central difference and
        whether it moves by at most switch_tol (relative) when every rotation's
        maximiser is held fixed, i.e. whether changes of maximiser within +-h
        (in rotations of any weight) leave the difference intact."""
        nk = self.coef.shape[0]
        fd = np.zeros(nk)
        ok = np.zeros(nk, bool)
        for k in range(nk):
            lp, lp_lin = self.losses(rot_mask, k, h, temperature, loss_fn)
            lm, lm_lin = self.losses(rot_mask, k, -h, temperature, loss_fn)
            fd[k] = (lp - lm) / (2 * h)
            fd_lin = (lp_lin - lm_lin) / (2 * h)
            ok[k] = abs(fd[k] - fd_lin) <= switch_tol * abs(fd[k])
        return fd, ok


def _lse(s, temperature):
    m = s.max()
    return m + temperature * np.log(np.exp((s - m) / temperature).sum())
