"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

from fluidmaxxer_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(inc, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(fm_\w+)\s*\(", text))
    return names


def test_header_declares_entry_points():
    names = declared_functions()
    assert "fm_step" in names and "fm_lattice_create" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_abi.LIBFM_PATH)
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_header():
    assert declared_functions() <= set(_abi.SIGNATURES), declared_functions() - set(_abi.SIGNATURES)


def test_abi_version_and_error_string():
    lib = _abi.lib()
    assert lib.fm_abi_version() == 1
    assert isinstance(lib.fm_last_error(), bytes)
