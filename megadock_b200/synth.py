"""Seeded synthetic protein generator for the docking workloads.

No benchmark structures are shipped with this project, so every workload is a
synthetic receptor/ligand pair written as ordinary PDB files that MEGADOCK's
reader accepts (src/pdb_entry.cpp:40-49: ATOM records, x/y/z in columns 31-54,
atom+residue name in columns 12-21, element in columns 77-78).

Recipe (per chain of n residues):
  * C-alpha trace: self-avoiding random walk with 3.8 A steps, confined to a
    sphere of radius 2.2 * n**(1/3) A; non-adjacent C-alphas stay >= 3.0 A apart.
  * Residue types drawn from natural amino-acid frequencies (UniProtKB/Swiss-Prot
    composition statistics, rounded to 0.01 %).
  * Heavy atoms with standard PDB names (which are CHARMM table keys such as
    "CA ALA"): backbone N, C, O around each C-alpha at ideal bond lengths
    (N-CA 1.46 A, CA-C 1.52 A, C=O 1.23 A) and side-chain atoms as a branched
    chain of 1.53 A bonds grown outward from the C-alpha.  About 7.8 heavy atoms
    per residue, so 150/70 residues give about 1,200/550 atoms.

Seeds: pair p of workload c uses seed 1000*c + p; receptor and ligand draw from
independent streams of that seed.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass

import numpy as np

# Natural amino-acid composition (percent).
AA_FREQ = {
    "ALA": 8.25, "ARG": 5.53, "ASN": 4.06, "ASP": 5.45, "CYS": 1.37,
    "GLN": 3.93, "GLU": 6.75, "GLY": 7.07, "HIS": 2.27, "ILE": 5.96,
    "LEU": 9.66, "LYS": 5.84, "MET": 2.42, "PHE": 3.86, "PRO": 4.70,
    "SER": 6.56, "THR": 5.34, "TRP": 1.08, "TYR": 2.92, "VAL": 6.87,
}

# Side-chain heavy atoms (standard PDB names) as (name, parent) pairs; the
# parent "CA" anchors the first atom.
SIDECHAIN = {
    "ALA": [("CB", "CA")],
    "ARG": [("CB", "CA"), ("CG", "CB"), ("CD", "CG"), ("NE", "CD"), ("CZ", "NE"), ("NH1", "CZ"), ("NH2", "CZ")],
    "ASN": [("CB", "CA"), ("CG", "CB"), ("OD1", "CG"), ("ND2", "CG")],
    "ASP": [("CB", "CA"), ("CG", "CB"), ("OD1", "CG"), ("OD2", "CG")],
    "CYS": [("CB", "CA"), ("SG", "CB")],
    "GLN": [("CB", "CA"), ("CG", "CB"), ("CD", "CG"), ("OE1", "CD"), ("NE2", "CD")],
    "GLU": [("CB", "CA"), ("CG", "CB"), ("CD", "CG"), ("OE1", "CD"), ("OE2", "CD")],
    "GLY": [],
    "HIS": [("CB", "CA"), ("CG", "CB"), ("ND1", "CG"), ("CD2", "CG"), ("CE1", "ND1"), ("NE2", "CD2")],
    "ILE": [("CB", "CA"), ("CG1", "CB"), ("CG2", "CB"), ("CD1", "CG1")],
    "LEU": [("CB", "CA"), ("CG", "CB"), ("CD1", "CG"), ("CD2", "CG")],
    "LYS": [("CB", "CA"), ("CG", "CB"), ("CD", "CG"), ("CE", "CD"), ("NZ", "CE")],
    "MET": [("CB", "CA"), ("CG", "CB"), ("SD", "CG"), ("CE", "SD")],
    "PHE": [("CB", "CA"), ("CG", "CB"), ("CD1", "CG"), ("CD2", "CG"), ("CE1", "CD1"), ("CE2", "CD2"), ("CZ", "CE1")],
    "PRO": [("CB", "CA"), ("CG", "CB"), ("CD", "CG")],
    "SER": [("CB", "CA"), ("OG", "CB")],
    "THR": [("CB", "CA"), ("OG1", "CB"), ("CG2", "CB")],
    "TRP": [("CB", "CA"), ("CG", "CB"), ("CD1", "CG"), ("CD2", "CG"), ("NE1", "CD1"), ("CE2", "CD2"),
            ("CE3", "CD2"), ("CZ2", "CE2"), ("CZ3", "CE3"), ("CH2", "CZ2")],
    "TYR": [("CB", "CA"), ("CG", "CB"), ("CD1", "CG"), ("CD2", "CG"), ("CE1", "CD1"), ("CE2", "CD2"),
            ("CZ", "CE1"), ("OH", "CZ")],
    "VAL": [("CB", "CA"), ("CG1", "CB"), ("CG2", "CB")],
}


@dataclass
class Chain:
    resnames: list
    atoms: list  # (name, resname, resseq, xyz(np.ndarray[3]))

    @property
    def coords(self) -> np.ndarray:
        return np.array([a[3] for a in self.atoms], dtype=np.float64)


def _unit(v):
    n = np.linalg.norm(v)
    return v / n if n > 0 else v


def _random_unit(rng):
    v = rng.normal(size=3)
    return v / np.linalg.norm(v)


def ca_walk(n: int, rng: np.random.Generator, step=3.8, min_sep=3.0, batch=64) -> np.ndarray:
    """Confined self-avoiding C-alpha walk.

    Each step draws `batch` candidate directions and keeps the first that stays
    inside the sphere and >= min_sep from every non-adjacent C-alpha.  A dead end
    backs the walk up three residues; every 50 dead ends the separation is
    relaxed by 5 %, so the walk always terminates (dense packing of the
    2.2 * n**(1/3) sphere is close to the jamming limit for 3.0 A)."""
    radius = 2.2 * n ** (1.0 / 3.0)
    pts = np.zeros((n, 3))
    m = 1
    dead_ends = 0
    while m < n:
        dirs = rng.normal(size=(batch, 3))
        dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
        cand = pts[m - 1] + step * dirs
        ok = np.linalg.norm(cand, axis=1) <= radius
        if m > 1:
            d = np.linalg.norm(cand[:, None, :] - pts[None, : m - 1, :], axis=2)
            ok &= d.min(axis=1) >= min_sep
        idx = np.flatnonzero(ok)
        if idx.size:
            pts[m] = cand[idx[0]]
            m += 1
        else:
            dead_ends += 1
            m = max(1, m - 3)
            if dead_ends % 50 == 0:
                min_sep *= 0.95
    return pts


def build_chain(n: int, rng: np.random.Generator) -> Chain:
    names = list(AA_FREQ)
    p = np.array([AA_FREQ[k] for k in names])
    p = p / p.sum()
    resnames = [names[i] for i in rng.choice(len(names), size=n, p=p)]
    ca = ca_walk(n, rng)
    centroid = ca.mean(axis=0)
    atoms = []
    for r in range(n):
        rn = resnames[r]
        prev_dir = _unit(ca[r - 1] - ca[r]) if r > 0 else _random_unit(rng)
        next_dir = _unit(ca[r + 1] - ca[r]) if r + 1 < n else _random_unit(rng)
        perp = _unit(np.cross(prev_dir, next_dir))
        if not np.any(perp):
            perp = _random_unit(rng)
        pos = {"CA": ca[r]}
        pos["N"] = ca[r] + 1.46 * _unit(prev_dir + 0.35 * perp)
        pos["C"] = ca[r] + 1.52 * _unit(next_dir - 0.35 * perp)
        pos["O"] = pos["C"] + 1.23 * _unit(-perp + 0.3 * _random_unit(rng))
        out_dir = _unit(ca[r] - centroid + 0.6 * _random_unit(rng))
        for name, parent in SIDECHAIN[rn]:
            d = _unit(out_dir + 0.7 * _random_unit(rng))
            pos[name] = pos[parent] + 1.53 * d
        order = ["N", "CA", "C", "O"] + [a for a, _ in SIDECHAIN[rn]]
        for name in order:
            atoms.append((name, rn, r + 1, pos[name]))
    return Chain(resnames, atoms)


def _element(name: str) -> str:
    return name[0]


def pdb_lines(chain: Chain, chain_id="A", offset=(0.0, 0.0, 0.0)):
    lines = []
    off = np.asarray(offset, dtype=np.float64)
    for i, (name, rn, seq, xyz) in enumerate(chain.atoms, start=1):
        x, y, z = xyz + off
        nm = f" {name:<3s}" if len(name) < 4 else name
        lines.append(
            f"ATOM  {i:5d} {nm:4s} {rn:3s} {chain_id:1s}{seq:4d}    "
            f"{x:8.3f}{y:8.3f}{z:8.3f}{1.0:6.2f}{0.0:6.2f}          {_element(name):>2s}  "
        )
    return lines


def write_pdb(path, chain: Chain, chain_id="A", offset=(0.0, 0.0, 0.0)):
    with open(path, "w") as f:
        f.write("REMARK  synthetic chain (megadock_b200.synth)\n")
        for ln in pdb_lines(chain, chain_id, offset):
            f.write(ln + "\n")
        f.write("END\n")


def make_pair(n_rec: int, n_lig: int, seed: int):
    """Receptor and ligand chains from independent streams of one seed."""
    ss = np.random.SeedSequence(seed)
    r_seed, l_seed = ss.spawn(2)
    rec = build_chain(n_rec, np.random.default_rng(r_seed))
    lig = build_chain(n_lig, np.random.default_rng(l_seed))
    return rec, lig


def write_pair(outdir, n_rec: int, n_lig: int, seed: int, stem: str | None = None):
    """Write <stem>_r.pdb and <stem>_l.pdb; returns their paths."""
    os.makedirs(outdir, exist_ok=True)
    stem = stem or f"syn{seed}"
    rec, lig = make_pair(n_rec, n_lig, seed)
    rp = os.path.join(outdir, f"{stem}_r.pdb")
    lp = os.path.join(outdir, f"{stem}_l.pdb")
    # the ligand is offset so the two files do not describe the same region
    write_pdb(rp, rec, "A", (10.0, -5.0, 3.0))
    write_pdb(lp, lig, "B", (40.0, 20.0, -12.0))
    return rp, lp


# Workloads (receptor residues, ligand residues, FFT N, rotation set, t).
WORKLOADS = {
    "plain-96": dict(n_rec=150, n_lig=70, nfft=96, rotations=3600, t=1, seed=0),
    "plain-128": dict(n_rec=500, n_lig=250, nfft=128, rotations=54000, t=3, seed=1000),
}


def smooth235(n: int) -> int:
    """Smallest 2^a 3^b 5^c >= n."""
    m = n
    while True:
        k = m
        for p in (2, 3, 5):
            while k % p == 0:
                k //= p
        if k == 1:
            return m
        m += 1


def uneven_pairs(npairs=64, seed_base=2000, lo=60, hi=800):
    """Pair list for the uneven-size batched workload: chain lengths log-uniform
    in [lo, hi] residues; returns (n_rec, n_lig, seed) per pair."""
    rng = np.random.default_rng(seed_base)
    out = []
    for p in range(npairs):
        a, b = np.exp(rng.uniform(math.log(lo), math.log(hi), size=2))
        out.append((int(round(max(a, b))), int(round(min(a, b))), seed_base + p))
    return out


# ---------------------------------------------------------------------------
# Planted complexes for fitting: a ligand rigidly placed in contact with the
# receptor surface, written in a rotated frame so that one rotation of the
# docking set and one grid translation restore the native placement exactly.

@dataclass
class PlantedComplex:
    rec_pdb: str
    lig_pdb: str
    rot_index: int             # rotation of the set that restores the native orientation
    shift: np.ndarray          # native translation in grid cells (signed)
    native_ca: np.ndarray      # native ligand C-alpha coordinates (receptor file frame)
    lig_file_ca: np.ndarray    # ligand C-alpha coordinates as written in the ligand file
    lig_ca_index: np.ndarray   # positions of the C-alphas in the ligand's heavy-atom list


def _bbox_mid(xyz):
    return (xyz.min(0) + xyz.max(0)) / 2


def _rounded(xyz):
    return np.round(np.asarray(xyz, np.float64), 3)


def decoy_ca(lig_file_ca, lig_center, rec_center, rotmat9, shift_signed, grid_width):
    """Ligand C-alphas of a docking pose: R (x - lig_center) - t * gw +
    rec_center, the placement a pose (rotation, translation t, t >= N/2 read
    as t - N) encodes (the score at t pairs receptor cell x with ligand cell
    x + t; both grids are centred on their molecule's bounding-box centre)."""
    m = np.asarray(rotmat9, np.float64).reshape(3, 3)
    return (np.asarray(lig_file_ca, np.float64) - lig_center) @ m.T - np.asarray(shift_signed) * grid_width + rec_center


def plant_complex(outdir, n_rec: int, n_lig: int, seed: int, rotation_set: int = 3600, grid_width: float = 1.2,
                  contact: float = 4.0, stem: str | None = None) -> PlantedComplex:
    """Receptor and ligand chains from `seed`; the ligand is moved along a
    seeded direction from the receptor centre until its closest heavy atom is
    `contact` A from the receptor (the native placement), then written
    rotated by the transpose of a seeded rotation of the docking set."""
    from scipy.spatial import cKDTree

    from ._native import data_dir, rotation_matrix
    os.makedirs(outdir, exist_ok=True)
    stem = stem or f"pl{seed}"
    rec, lig = make_pair(n_rec, n_lig, seed)
    rng = np.random.default_rng(np.random.SeedSequence(seed).spawn(3)[2])
    rec_xyz = np.array([a[3] for a in rec.atoms])
    lig_xyz = np.array([a[3] for a in lig.atoms])
    lig_xyz = lig_xyz - lig_xyz.mean(0)
    tree = cKDTree(rec_xyz)
    u = _random_unit(rng)
    centre = rec_xyz.mean(0)
    lo, hi = 0.0, 400.0                      # distance along u: overlap at lo, apart at hi
    for _ in range(60):
        mid = (lo + hi) / 2
        d, _ = tree.query(lig_xyz + centre + mid * u)
        if d.min() < contact:
            lo = mid
        else:
            hi = mid
    native = lig_xyz + centre + hi * u
    angles = np.fromfile(os.path.join(data_dir(), f"rotations_{rotation_set}.f32"), np.float32).reshape(-1, 3)
    k = int(rng.integers(len(angles)))
    m = rotation_matrix(angles[k]).astype(np.float64).reshape(3, 3)
    file_xyz = _rounded((native - native.mean(0)) @ m + np.array([40.0, 20.0, -12.0]))
    rec_file = _rounded(rec_xyz)
    rec_c = _bbox_mid(rec_file.astype(np.float32).astype(np.float64))
    lig_c = _bbox_mid(file_xyz.astype(np.float32).astype(np.float64))
    ca = np.array([i for i, a in enumerate(lig.atoms) if a[0] == "CA"])
    placed = decoy_ca(file_xyz, lig_c, rec_c, m.reshape(-1), np.zeros(3), grid_width)
    shift = np.round((placed - native).mean(0) / grid_width).astype(np.int64)
    native_ca = decoy_ca(file_xyz[ca], lig_c, rec_c, m.reshape(-1), shift, grid_width)
    rp = os.path.join(outdir, f"{stem}_r.pdb")
    lp = os.path.join(outdir, f"{stem}_l.pdb")
    write_pdb(rp, Chain(rec.resnames, [(a[0], a[1], a[2], x) for a, x in zip(rec.atoms, rec_file)]), "A")
    write_pdb(lp, Chain(lig.resnames, [(a[0], a[1], a[2], x) for a, x in zip(lig.atoms, file_xyz)]), "B")
    return PlantedComplex(rp, lp, k, shift, native_ca, file_xyz[ca], ca)


def fitting_pairs(npairs=32, seed_base=4000, lo=200, hi=1500):
    """(n_rec, n_lig, seed) of the fitting workload: chain lengths log-uniform
    in [lo, hi] residues, seed = seed_base + pair index."""
    rng = np.random.default_rng(seed_base)
    out = []
    for p in range(npairs):
        n_rec, n_lig = np.exp(rng.uniform(np.log(lo), np.log(hi), 2)).astype(int)
        out.append((int(n_rec), int(n_lig), seed_base + p))
    return out
