"""The C ABI library loads and exports every entry point include/md_b200.h declares."""
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _declared():
    text = (ROOT / "include" / "md_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(md_[a-z0-9_]+)\s*\(", text)))


def test_header_matches_binding(built):
    from megadock_b200 import _native
    assert _declared() == _native.EXPORTED


def test_library_exports_all_symbols(built):
    import ctypes
    from megadock_b200 import _native
    L = ctypes.CDLL(str(_native.LIB_PATH))
    missing = [s for s in _declared() if not hasattr(L, s)]
    assert not missing, missing


def test_cli_built(built):
    from megadock_b200 import _native
    assert _native.CLI_PATH.exists()


def test_kernel_sizes_built(built):
    from megadock_b200 import lib
    for n in (32, 36, 40, 44, 48, 56, 60, 64, 72, 80, 84, 88, 96, 100, 108, 112, 120, 128, 132, 140, 144, 160,
              42, 50, 54, 66, 70, 90, 98, 110, 126, 150, 154,
              162, 168, 176, 180, 192, 196, 198, 200, 210, 216, 220, 224,
              # staged sizes: every 2 ng1 of the default grid table up to ng1 = 160
              240, 242, 250, 252, 256, 264, 270, 280, 288, 294, 300, 308, 320,
              324, 330, 336, 350, 352, 360, 378, 384, 392, 396, 400, 420, 432, 440,
              448, 450, 462, 480, 484, 486, 490, 500, 504, 512):
        assert lib().md_fft_size_supported(n) == 1
    for n in (46, 230, 244, 520, 1024, 2048):
        assert lib().md_fft_size_supported(n) == 0


def test_staged_sizes_cover_the_default_table(built):
    """Every FFT edge 2 ng1 of the default (-l 11) grid table with ng1 in
    (112, 256] has a kernel set, so automatic sizing never stops below 512."""
    from pathlib import Path

    from megadock_b200 import lib
    tables = Path(__file__).resolve().parent.parent / "megadock_b200" / "data" / "fft_tables.tsv"
    row = [l.split("\t")[1].split() for l in tables.read_text().splitlines() if l.split("\t")[0] == "11"][0]
    for ng1 in map(int, row):
        if 112 < ng1 <= 256:
            assert lib().md_fft_size_supported(2 * ng1) == 1, 2 * ng1


def test_null_arguments_are_rejected(built):
    """Entry points check their pointers before touching a device (no GPU needed)."""
    import ctypes as C

    from megadock_b200 import _native as N
    L = N.lib()
    E = N.MD_ERR_ARG
    f = C.POINTER(C.c_float)()
    assert L.md_adjoint_lse(None, f, 1, None, 10.0, 1.0, None, f, f, f, None, None, 0, f, f) == E
    assert L.md_adjoint_poses(None, f, 1, None, f, f, f, f, None, 0, f, f) == E
    assert L.md_pose_scores(None, f, 1, None, f) == E
    assert L.md_release_work(None) == E
    assert L.md_set_lanes(None, 1) == E
    assert L.md_pose_terms(None, f, f, 1, None, f) == E
    assert L.md_receptor_build(None, 1, f, f, f, f, -45.0, 1.0, 1.0, 1, f, f) == E
    assert L.md_job_receptor_to(None, None) == E
    assert L.md_job_write_out(None, None, None, 0) == E
    assert L.md_decoy_pdb(None, None, 1, None) == E
    assert L.md_ligand_centres(None, 0, None) == E
    assert L.md_decoy_pdb(b"/nonexistent.out", b"/nonexistent.pdb", 1, b"/tmp/x.pdb") == N.MD_ERR_IO
