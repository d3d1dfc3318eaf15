"""The C-ABI library loads, exports every symbol include/weno_sb.h declares,
and rejects bad arguments before touching a GPU.  CPU only."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def L():
    from wenostandalone_b200 import _lib, build
    build.build_lib()
    _lib.lib()
    return _lib


def declared_functions():
    txt = open(os.path.join(ROOT, "include", "weno_sb.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(weno_sb_\w+)\s*\(", txt)))


def test_every_declared_symbol_is_exported(L):
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (weno_sb_\w+)", out))
    decl = declared_functions()
    assert decl, "no declarations found"
    missing = [f for f in decl if f not in exported]
    assert not missing, missing
    # and the Python binding knows all of them
    assert sorted(L.EXPORTED) == decl


def test_version_and_extents(L):
    lib = L.lib()
    assert lib.weno_sb_version() == 1
    g = L.WenoGrid(199, 99, 49, 8, 6, 0, 1e-16, 1e-5)
    ns, c1, c2 = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
    for d, exp in enumerate([(212, 112, 62), (112, 212, 62), (62, 112, 212)]):
        assert lib.weno_sb_extents(ctypes.byref(g), d, ctypes.byref(ns), ctypes.byref(c1), ctypes.byref(c2)) == 0
        assert (ns.value, c1.value, c2.value) == exp


@pytest.mark.parametrize("field,val,needle", [
    ("v_size", 0, "v_size"), ("buff_size", 2, "buff_size"), ("m_cells", -1, "negative"),
    ("scheme", 9, "scheme")])
def test_grid_validation(L, field, val, needle):
    lib = L.lib()
    g = L.WenoGrid(15, 15, 15, 2, 6, 0, 1e-16, 1e-5)
    setattr(g, field, val)
    h = ctypes.c_int(0)
    assert lib.weno_sb_init(ctypes.byref(g), 0, ctypes.byref(h)) == L.ERR_ARG
    assert needle in L.last_error()


def test_bad_direction_and_handle(L):
    lib = L.lib()
    g = L.WenoGrid(15, 15, 15, 2, 6, 0, 1e-16, 1e-5)
    assert lib.weno_sb_extents(ctypes.byref(g), 3, None, None, None) == L.ERR_ARG
    assert lib.weno_sb_weno(12345, 0, 5, 0) == L.ERR_HANDLE
    assert lib.weno_sb_sync(0) == L.ERR_HANDLE
    assert lib.weno_sb_finalize(-1) == L.ERR_HANDLE


def test_fault_injection_is_host_side(L, monkeypatch):
    """WENO_SB_FAULT makes the named operation fail before any CUDA call."""
    lib = L.lib()
    g = L.WenoGrid(15, 15, 15, 2, 6, 0, 1e-16, 1e-5)
    monkeypatch.setenv("WENO_SB_FAULT", "upload,init")
    h = ctypes.c_int(0)
    assert lib.weno_sb_init(ctypes.byref(g), 0, ctypes.byref(h)) == L.ERR_INJECTED
    assert "init" in L.last_error()
    monkeypatch.setenv("WENO_SB_FAULT", "launch")
    rc = lib.weno_sb_reshape_dev(ctypes.byref(g), 0, 0, 1, 1, None)
    assert rc == L.ERR_INJECTED


def test_flag_validation(L):
    lib = L.lib()
    g = L.WenoGrid(15, 15, 15, 2, 6, 0, 1e-16, 1e-5)
    cf = L.WenoCoefs(8, 8, 8, 8, 8)
    rc = lib.weno_sb_weno_dev(ctypes.byref(g), 0, 5, 1 << 7, 0, 8, ctypes.byref(cf), 8, 8, None)
    assert rc == L.ERR_ARG and "flag" in L.last_error()
    rc = lib.weno_sb_weno_dev(ctypes.byref(g), 0, 5, 0, 0, None, ctypes.byref(cf), 8, 8, None)
    assert rc == L.ERR_ARG and "NULL" in L.last_error()
