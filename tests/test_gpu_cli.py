"""The command line end to end (GPU): megadock-b200 writes the same .out as
the reference's own program for the same flags (scores within 1e-4 relative;
pose lines compared as a multiset at ties)."""
import subprocess

import numpy as np
import pytest

from conftest import needs_ref

pytestmark = pytest.mark.gpu


def _parse(path):
    lines = open(path).read().splitlines()
    head = lines[:4]
    poses = [l.split("\t") for l in lines[4:]]
    rec = np.array([(float(p[0]), float(p[1]), float(p[2]), int(p[3]), int(p[4]), int(p[5]), float(p[6]))
                    for p in poses])
    return head, rec


def test_cli_writes_out_file(built, gpu, pairs, tmp_path):
    from megadock_b200 import _native
    rp, lp = pairs["small"]
    out = tmp_path / "x.out"
    res = subprocess.run([str(_native.CLI_PATH), "-R", rp, "-L", lp, "-F", "64", "-r", "360", "-N", "50",
                          "-o", str(out)], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    head, rec = _parse(out)
    assert head[0] == "64\t1.20"
    assert head[1] == "\t0.000000\t0.000000\t0.000000"
    assert len(rec) == 50
    assert (np.diff(rec[:, 6]) <= 0).all()


def test_cli_usage_error(built):
    from megadock_b200 import _native
    res = subprocess.run([str(_native.CLI_PATH), "-L", "x.pdb"], capture_output=True, text=True)
    assert res.returncode != 0


@needs_ref
def test_cli_matches_reference_out(built, gpu, pairs, tmp_path):
    from megadock_b200 import _native
    from oracle.ref import REF_BIN
    rp, lp = pairs["c0"]
    flags = ["-R", rp, "-L", lp, "-F", "96", "-e", "0.06", "-r", "360", "-t", "2", "-N", "300"]
    ours, theirs = tmp_path / "ours.out", tmp_path / "ref.out"
    r1 = subprocess.run([str(_native.CLI_PATH), *flags, "-o", str(ours)], capture_output=True, text=True)
    assert r1.returncode == 0, r1.stderr
    r2 = subprocess.run([str(REF_BIN), *flags, "-o", str(theirs)], capture_output=True, text=True)
    assert r2.returncode == 0
    h1, a = _parse(ours)
    h2, b = _parse(theirs)
    assert h1 == h2
    assert len(a) == len(b)
    # scores rank-by-rank within tolerance
    np.testing.assert_allclose(a[:, 6], b[:, 6], rtol=1e-4, atol=0.011)
    # pose identity: every reference pose whose score is clear of its
    # neighbours (no near tie) appears in ours with the same angles and cell
    ours_set = {tuple(np.round(x[:6], 6)) for x in a}
    gaps = np.abs(np.diff(b[:, 6]))
    for n in range(1, len(b) - 1):
        if gaps[n - 1] > 0.05 and gaps[n] > 0.05:
            assert tuple(np.round(b[n, :6], 6)) in ours_set, b[n]


@needs_ref
def test_cli_automatic_size_above_224(built, gpu, pairs, tmp_path):
    """Automatic grid sizing that lands above FFT edge 224 (the 500/250-residue
    pair at grid width 0.55 A needs ng1 = 120, N = 240): the device receptor
    build and the staged kernels give the reference's .out."""
    from megadock_b200 import _native
    from oracle.ref import REF_BIN
    rp, lp = pairs["c1"]
    flags = ["-R", rp, "-L", lp, "-v", "0.55", "-r", "24", "-t", "2", "-N", "40"]
    ours, theirs = tmp_path / "ours.out", tmp_path / "ref.out"
    r1 = subprocess.run([str(_native.CLI_PATH), *flags, "-o", str(ours)], capture_output=True, text=True)
    assert r1.returncode == 0, r1.stderr
    r2 = subprocess.run([str(REF_BIN), *flags, "-o", str(theirs)], capture_output=True, text=True)
    assert r2.returncode == 0
    h1, a = _parse(ours)
    h2, b = _parse(theirs)
    assert h1 == h2
    assert h1[0].startswith("240\t")
    np.testing.assert_allclose(a[:, 6], b[:, 6], rtol=1e-4, atol=0.011)
    ours_set = {tuple(np.round(x[:6], 6)) for x in a}
    gaps = np.abs(np.diff(b[:, 6]))
    for n in range(1, len(b) - 1):
        if gaps[n - 1] > 0.05 and gaps[n] > 0.05:
            assert tuple(np.round(b[n, :6], 6)) in ours_set, b[n]


@needs_ref
def test_cli_large_receptor_automatic_size(built, gpu, tmp_path):
    """A 2,000-residue synthetic receptor with a 250-residue ligand, the grid
    size chosen automatically from the reference's table (no -F): the command
    line docks it and writes the reference's .out."""
    from megadock_b200 import _native, synth
    from oracle.ref import REF_BIN
    rp, lp = synth.write_pair(str(tmp_path), 2000, 250, 7, stem="big")
    flags = ["-R", rp, "-L", lp, "-r", "24", "-t", "2", "-N", "40"]
    ours, theirs = tmp_path / "ours.out", tmp_path / "ref.out"
    r1 = subprocess.run([str(_native.CLI_PATH), *flags, "-o", str(ours)], capture_output=True, text=True)
    assert r1.returncode == 0, r1.stderr
    r2 = subprocess.run([str(REF_BIN), *flags, "-o", str(theirs)], capture_output=True, text=True)
    assert r2.returncode == 0
    h1, a = _parse(ours)
    h2, b = _parse(theirs)
    assert h1 == h2
    np.testing.assert_allclose(a[:, 6], b[:, 6], rtol=1e-4, atol=0.011)
    ours_set = {tuple(np.round(x[:6], 6)) for x in a}
    gaps = np.abs(np.diff(b[:, 6]))
    for n in range(1, len(b) - 1):
        if gaps[n - 1] > 0.05 and gaps[n] > 0.05:
            assert tuple(np.round(b[n, :6], 6)) in ours_set, b[n]
