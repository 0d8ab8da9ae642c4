"""The C-ABI library loads and exports every entry point declared in
include/bem200.h (no device work)."""
import os
import re

from conftest import ROOT


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "bem200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bem200_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "bem200_green_assemble" in syms and "bem200_last_error" in syms


def test_library_exports_all_declared_symbols():
    from mnpbem_b200 import _native
    lib = _native.lib()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_version_and_error_string():
    from mnpbem_b200 import _native
    assert _native.lib().bem200_version() >= 100
    # an argument error is reported without touching the device
    st = _native.lib().bem200_refine_count(0, None, None, 0.0, 3.0, None, None)
    assert st == 1
    assert "refine_count" in _native.last_error()


def test_every_declared_symbol_has_a_ctypes_signature():
    """Calls through mnpbem_b200._native use explicit argument types (doubles
    and 64-bit sizes would be mangled by ctypes' defaults)."""
    from mnpbem_b200 import _native
    missing = [s for s in declared_symbols() if s not in _native._SIGS]
    assert not missing, missing
