"""The .out consumers on the CPU: decoygen (decoy complex of one pose) and
calcrg (placed ligand centres) give byte-identical output to the reference's
own tools, built from their sources under oracle/_ref, on a .out written by
the reference's program and on a synthetic .out with wrapped translations."""
import subprocess

import numpy as np
import pytest

from conftest import needs_ref


def _bin(name):
    from megadock_b200 import _native
    return str(_native.CLI_PATH.parent / name)


def _synthetic_out(path, lig_pdb, rec_pdb, n=64, seed=3):
    rng = np.random.default_rng(seed)
    lines = [f"{n}\t1.20", "\t0.000000\t0.000000\t0.000000", f"{rec_pdb}\t10.632000\t-5.847000\t4.284500",
             f"{lig_pdb}\t40.556499\t19.870001\t-14.546499"]
    for _ in range(40):
        a = rng.uniform(-np.pi, np.pi, 3)
        t = rng.integers(0, n, 3)
        lines.append(f"{a[0]:f}\t{a[1]:f}\t{a[2]:f}\t{t[0]}\t{t[1]}\t{t[2]}\t{rng.uniform(0, 3000):.2f}")
    path.write_text("\n".join(lines) + "\n")


@needs_ref
def test_decoygen_and_calcrg_match_reference(built, pairs, tmp_path):
    from oracle.ref import REF_BIN
    rp, lp = pairs["small"]
    real = tmp_path / "real.out"
    r = subprocess.run([str(REF_BIN), "-R", rp, "-L", lp, "-F", "64", "-r", "24", "-N", "20", "-o", str(real)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    syn = tmp_path / "syn.out"
    _synthetic_out(syn, lp, rp)
    refdir = REF_BIN.parent
    for out, decoys in ((real, (1, 2, 20)), (syn, (1, 7, 40))):
        for d in decoys:
            a, b = tmp_path / f"ours_{d}.pdb", tmp_path / f"ref_{d}.pdb"
            assert subprocess.run([_bin("decoygen"), str(a), lp, str(out), str(d)]).returncode == 0
            subprocess.run([str(refdir / "decoygen"), str(b), lp, str(out), str(d)], check=True)
            assert a.read_bytes() == b.read_bytes(), (out.name, d)
        for mode in ("0", "1"):
            x = subprocess.run([_bin("calcrg"), str(out), mode], capture_output=True, check=True).stdout
            y = subprocess.run([str(refdir / "calcrg"), str(out), mode], capture_output=True, check=True).stdout
            assert x == y and len(x) > 0


def test_tool_usage(built):
    r = subprocess.run([_bin("decoygen")], capture_output=True, text=True)
    assert r.returncode == 255 and "decoygen" in r.stdout
    r = subprocess.run([_bin("calcrg")], capture_output=True, text=True)
    assert r.returncode == 255 and "center points" in r.stdout
