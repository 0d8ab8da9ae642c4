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


def test_inverse_nopiv_argument_errors_without_device_work():
    """bem200_inverse_nopiv rejects bad sizes, a leading dimension other than n
    and an unknown dtype before any device call (fake non-null pointers are
    never touched)."""
    import ctypes
    from mnpbem_b200 import _native
    lib = _native.lib()
    fake = ctypes.c_void_p(256)
    info = ctypes.cast(ctypes.c_void_p(512), ctypes.POINTER(ctypes.c_int32))
    st = lib.bem200_inverse_nopiv(_native.C64, 0, 0, fake, 0, None, 0, fake, 1e-2, info, None)
    assert st == 1 and "inverse_nopiv" in _native.last_error()
    st = lib.bem200_inverse_nopiv(_native.C64, 0, 64, fake, 65, None, 0, fake, 1e-2, info, None)
    assert st == 4 and "ld" in _native.last_error()
    st = lib.bem200_inverse_nopiv(99, 0, 64, fake, 64, None, 0, fake, 1e-2, info, None)
    assert st == 1 and "dtype" in _native.last_error()


def test_inverse_nopiv_scratch_sizes():
    """The scratch of the no-pivot inverse: none for a bad size or dtype, twice
    the complex64 bytes for complex128, and for n = 2 m about what the two
    live Schur blocks of the top level (2 m^2 elements) plus the recursion
    below need."""
    from mnpbem_b200 import _native
    lib = _native.lib()
    assert lib.bem200_inverse_nopiv_workspace_size(_native.C64, 0) == 0
    assert lib.bem200_inverse_nopiv_workspace_size(99, 1000) == 0
    for n in (64, 200, 1000, 5768):
        s64 = lib.bem200_inverse_nopiv_workspace_size(_native.C64, n)
        s128 = lib.bem200_inverse_nopiv_workspace_size(_native.C128, n)
        assert s128 - 256 == 2 * (s64 - 256)
        assert s64 >= 8 * 3 * n
    m = 2944
    s = lib.bem200_inverse_nopiv_workspace_size(_native.C64, 2 * m)
    assert 8 * 2 * m * m < s < 8 * 3 * m * m
