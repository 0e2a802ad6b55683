"""The C-ABI library loads and exports every entry point that include/cufil.h declares (no GPU needed)."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "cufil.h").read_text()
    return sorted(set(re.findall(r"CF_API\s+[\w\s\*]*?\b(cf_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "cf_mobility_create" in names and "cf_apply_mobility" in names and "cf_sim_step" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol():
    from cufcm_fil_b200 import _lib
    L = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, missing


def test_bindings_cover_header():
    from cufcm_fil_b200 import _lib
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_version_and_error_text_without_gpu():
    from cufcm_fil_b200 import _lib
    L = _lib.load()
    assert L.cf_version() >= 10000
    # Invalid arguments are rejected on the host before any CUDA call.
    cfg = _lib.MobilityConfig(0, 0, 1, 3, 1.0, 1.0, 1.0, 0)
    h = ctypes.c_void_p()
    rc = L.cf_mobility_create(ctypes.byref(cfg), ctypes.byref(h))
    assert rc == _lib.CF_EINVAL
    assert "n_seg + n_blob" in _lib.last_error()
    cfg = _lib.MobilityConfig(10, 0, 1, 4, 1.0, 1.0, 1.0, 0)
    assert L.cf_mobility_create(ctypes.byref(cfg), ctypes.byref(h)) == _lib.CF_EINVAL
