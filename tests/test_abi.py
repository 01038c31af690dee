"""The C-ABI library builds, loads and exports every entry point declared in
include/sawsim_b200.h (no compute calls: no GPU needed)."""
import ctypes
import re

from conftest import REPO


def declared():
    txt = (REPO / 'include' / 'sawsim_b200.h').read_text()
    return sorted(set(re.findall(r'\b(ss_[a-z0-9_]+)\s*\(', txt)))


def test_header_and_binding_agree():
    from sawsim_b200 import _lib
    assert declared() == sorted(n for n, _, _ in _lib.SIGNATURES)


def test_library_exports_all(built_lib):
    lib = ctypes.CDLL(str(built_lib))
    for name in declared():
        assert hasattr(lib, name), name


def test_python_binding_loads(built_lib):
    from sawsim_b200 import _lib
    lib = _lib.load()
    assert lib.ss_last_error(None) == b'null handle'
