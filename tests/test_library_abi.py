"""CPU tests of the C ABI boundary: the library loads and exports exactly the
entry points include/xcal_b200.h declares (no compute calls without a GPU)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "xcal_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(xcal_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "xcal_simple_iterate" in syms and "xcal_case_create" in syms
    assert len(syms) >= 30


def test_library_exports_every_declared_symbol(x):
    from importlib import import_module
    lib_mod = import_module("xcalibre_b200._lib")
    L = ctypes.CDLL(lib_mod.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing
    # the Python binding declares a signature for every entry point
    assert sorted(lib_mod.SIGNATURES) == declared_symbols()


def test_version_string(x):
    from importlib import import_module
    v = import_module("xcalibre_b200._lib").lib().xcal_version().decode()
    assert "sm_100a" in v


def test_ctx_create_fails_cleanly_without_gpu(x):
    import torch
    if torch.cuda.is_available():
        return
    from importlib import import_module
    L = import_module("xcalibre_b200._lib").lib()
    h = ctypes.c_void_p()
    assert L.xcal_ctx_create(0, ctypes.byref(h)) != 0
    assert not h.value


def test_oracle_library_loads(orc):
    assert orc.threads() >= 1
