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
    for n in (32, 48, 64, 72, 80, 96, 100, 108, 112, 120, 128, 144, 160):
        assert lib().md_fft_size_supported(n) == 1
    for n in (90, 98, 2048):
        assert lib().md_fft_size_supported(n) == 0
