"""Detail output (-O) on the GPU against the reference's own program: the
.detail header and the block around the input placement are identical text,
and every docking-result row whose pose both programs found (same angles and
translation) carries identical score terms, RMSD and near-native flag
(src/docking.cpp:456-898)."""
import subprocess

import pytest

from conftest import needs_ref

pytestmark = pytest.mark.gpu


def _rows(lines):
    out = {}
    for ln in lines:
        rank, rest = ln.split(":", 1)
        key = rest[:36]                  # "(angles) (trans)"
        out.setdefault(key, rest)
    return out


@needs_ref
@pytest.mark.parametrize("name,flags", [("small", ["-F", "64", "-r", "360", "-N", "60"]),
                                        ("c0", ["-F", "96", "-r", "360", "-N", "80", "-e", "0.5"])])
def test_detail_matches_reference(built, gpu, pairs, tmp_path, name, flags):
    from megadock_b200 import _native
    from oracle.ref import REF_BIN
    rp, lp = pairs[name]
    args = ["-R", rp, "-L", lp, *flags, "-O"]
    ours, theirs = tmp_path / "ours.out", tmp_path / "ref.out"
    r1 = subprocess.run([str(_native.CLI_PATH), *args, "-o", str(ours)], capture_output=True, text=True)
    assert r1.returncode == 0, r1.stderr
    r2 = subprocess.run([str(REF_BIN), *args, "-o", str(theirs)], capture_output=True, text=True)
    assert r2.returncode == 0
    a = (tmp_path / "ours.detail").read_text().splitlines()
    b = (tmp_path / "ref.detail").read_text().splitlines()
    assert len(a) == len(b)
    cut = a.index(" *** docking results *** ")
    assert a[:cut] == b[:cut]
    ra, rb = _rows(a[cut + 3:]), _rows(b[cut + 3:])
    common = set(ra) & set(rb)
    assert len(common) >= 0.9 * len(rb)
    for k in common:
        assert ra[k] == rb[k], (k, ra[k], rb[k])
    ca = (tmp_path / "ours.csv").read_text().splitlines()
    cb = (tmp_path / "ref.csv").read_text().splitlines()
    assert ca[0] == cb[0] and len(ca) == len(cb)
    ka = {",".join(x.split(",")[1:7]): x.split(",", 1)[1] for x in ca[1:]}
    kb = {",".join(x.split(",")[1:7]): x.split(",", 1)[1] for x in cb[1:]}
    for k in set(ka) & set(kb):
        assert ka[k] == kb[k]
