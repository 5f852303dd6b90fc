"""CPU checks of the C ABI library: it builds/loads and exports every entry
point declared in include/cmmdft_b200.h (no compute calls without a GPU)."""
import ctypes
import os
import re

from cmmdft_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "cmmdft_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cmm_[a-z0-9_]+)\s*\(", src)))


def test_library_loads_and_exports_header_symbols():
    lib = _lib.lib()
    names = declared_symbols()
    assert len(names) >= 12
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) <= set(_lib.exported_symbols()) | set(names)


def test_version_and_status_strings():
    lib = _lib.lib()
    assert lib.cmm_version() >= 100
    assert lib.cmm_status_string(0) == b"ok"
    assert b"shared memory" in lib.cmm_status_string(4)


def test_bindings_cover_header():
    assert set(declared_symbols()) == set(_lib.exported_symbols())
