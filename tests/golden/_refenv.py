"""Import helper for the reference ``mnpbem`` package (fixture generation only).

The reference imports matplotlib / mpl_toolkits / tqdm at module level for
plotting, and none of them is installed here.  This helper registers
import-only stand-in modules for those names, points numba's cache at a
writable directory and puts the read-only reference checkout on sys.path.
It is used only by ``make_golden.py`` in this directory, which runs in the
build container where the reference checkout exists.
"""
import importlib.abc
import importlib.machinery
import os
import sys
import types

REFERENCE_ROOT = os.environ.get("MNPBEM_REFERENCE")
if not REFERENCE_ROOT:
    raise RuntimeError("set MNPBEM_REFERENCE to the path of the reference checkout to generate fixtures")
_STUB_ROOTS = ("matplotlib", "mpl_toolkits", "tqdm")


class _Anything(types.ModuleType):
    """Module whose every attribute is a callable no-op object."""

    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        return _Dummy()


class _Dummy:
    def __call__(self, *a, **k):
        return _Dummy()

    def __getattr__(self, name):
        return _Dummy()

    def __iter__(self):
        return iter(())

    def __mro_entries__(self, bases):
        return (object,)


class _StubFinder(importlib.abc.MetaPathFinder, importlib.abc.Loader):
    def find_spec(self, fullname, path, target=None):
        if fullname.split(".")[0] in _STUB_ROOTS:
            return importlib.machinery.ModuleSpec(fullname, self, is_package=True)
        return None

    def create_module(self, spec):
        m = _Anything(spec.name)
        m.__path__ = []
        return m

    def exec_module(self, module):
        pass


def setup():
    if not any(isinstance(f, _StubFinder) for f in sys.meta_path):
        sys.meta_path.insert(0, _StubFinder())
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache_ref")
    os.environ.setdefault("MNPBEM_GPU", "0")
    if REFERENCE_ROOT not in sys.path:
        sys.path.insert(0, REFERENCE_ROOT)
    import mnpbem  # noqa: F401
    return mnpbem
