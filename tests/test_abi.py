"""The C-ABI library: it loads without a GPU and exports every entry point include/isw.h declares. CPU only (no compute
calls are made here)."""
import ctypes
import re

from conftest import ROOT, PKG


def declared():
    text = (ROOT / 'include' / 'isw.h').read_text()
    return re.findall(r'^\s*(?:int|const char \*)\s*(isw_\w+)\s*\(', text, re.M)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(PKG / 'isw' / 'libisw.so'))
    names = declared()
    assert len(names) >= 14
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    lib.isw_version.restype = ctypes.c_int
    assert lib.isw_version() >= 100


def test_library_has_no_dynamic_cuda_runtime():
    """The CUDA runtime is linked statically: the library depends on the driver only, not on a libcudart copy."""
    import subprocess
    out = subprocess.run(['ldd', str(PKG / 'isw' / 'libisw.so')], capture_output=True, text=True).stdout
    assert 'libcudart' not in out


def test_python_facade_binds_every_symbol():
    from isw import _lib
    for n in declared():
        assert hasattr(_lib, n), n
