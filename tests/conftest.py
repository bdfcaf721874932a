"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU.

Inputs are synthetic PDB pairs from megadock_b200.synth (seeded, written to a
temporary directory per session).  Parity checkers: the reference compiled from
its own sources (oracle/_ref, when built) and the oracle restatement
(oracle/md_oracle.c + numpy FFTs).
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_built():
    from megadock_b200 import _native
    if not _native.LIB_PATH.exists():
        from megadock_b200.build import build
        build()
    import subprocess
    from oracle import oracle as O
    if not O.LIB.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "restatement"], check=True, capture_output=True)


@pytest.fixture(scope="session")
def built():
    _ensure_built()
    return True


@pytest.fixture(scope="session")
def pairs(tmp_path_factory):
    """Synthetic receptor/ligand PDB pairs keyed by name."""
    from megadock_b200 import synth
    d = tmp_path_factory.mktemp("pdb")
    out = {}
    for name, (nr, nl, seed) in {
        "c0": (150, 70, 0),        # 96^3 workload pair
        "c1": (500, 250, 1000),    # 128^3 workload pair
        "small": (30, 16, 8),      # 64^3 quick pair
    }.items():
        out[name] = synth.write_pair(str(d), nr, nl, seed, stem=name)
    return out


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not has_gpu():
        pytest.skip("no CUDA device")
    return 0


def ref_available():
    from oracle import ref
    return ref.available()


needs_ref = pytest.mark.skipif(not ref_available(), reason="reference build (oracle/_ref) not present")
