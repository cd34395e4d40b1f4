"""The C-ABI library loads without a GPU and exports every entry point that
include/hrdaya_b200.h declares (no compute calls here)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(hp_[a-z0-9_]+)\s*\(", txt))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "hp_mono_create" in names and "hp_last_error" in names


def test_library_exports_all_declared_symbols():
    from hrdayapy_b200 import _lib
    L = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, missing


def test_version_and_error_without_gpu():
    from hrdayapy_b200 import _lib
    L = _lib.lib()
    assert b"sm_100a" in L.hp_version()
    # argument validation happens before any device call
    h = ctypes.c_void_p()
    st = L.hp_mono_create(None, ctypes.byref(h), None)
    assert st == 1
    assert b"null" in L.hp_last_error()
