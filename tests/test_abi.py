"""The C-ABI library loads without a GPU and exports every symbol that include/*.h declares."""
import ctypes
import os
import re

from discrete_adjoint_b200 import _ffi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if not f.endswith(".h"):
            continue
        src = open(os.path.join(inc, f)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"\b(da_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_library_loads_and_exports_all_declared_symbols():
    lib = _ffi.load()
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    # every declared symbol also has a ctypes signature bound
    assert names <= set(_ffi.SIGNATURES), sorted(names - set(_ffi.SIGNATURES))


def test_abi_version_and_strerror():
    lib = _ffi.load()
    assert lib.da_abi_version() == 2
    assert lib.da_strerror(_ffi.DA_ERR_NAN) == b"non-finite state or time step"
    assert lib.da_strerror(12345) == b"unknown error"


def test_create_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        return
    lib = _ffi.load()
    p = _ffi.da_params()
    lib.da_params_default(ctypes.byref(p))
    err = ctypes.c_int(0)
    ctx = lib.da_create(ctypes.byref(p), ctypes.byref(err))
    assert not ctx and err.value == _ffi.DA_ERR_NO_DEVICE


def test_params_default_matches_reference_constants():
    lib = _ffi.load()
    p = _ffi.da_params()
    lib.da_params_default(ctypes.byref(p))
    assert p.frict_tiny_iters == 50 and p.frict_tiny_early == 0.1 and p.frict_tiny_late == 1e-9
    assert p.gamma == 1.0 and p.epsilon == 1.0
    assert abs(p.intfrict - 30 * 3.1415926 / 180) < 1e-15
