"""The C ABI library loads and exports every symbol its headers declare (no GPU needed)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include")))
           if f.endswith(".h")]


def declared():
    names = set()
    for h in HEADERS:
        with open(h) as f:
            src = f.read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[\w\s\*]+?\b(rls_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_entry_points():
    names = declared()
    assert "rls_pstrirecy_schur" in names and "rls_grid_zigzag" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol(built_lib):
    lib = C.CDLL(built_lib)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header(built_lib):
    from rls_b200._lib import SIGNATURES
    assert set(declared()) == set(SIGNATURES)


def test_status_strings_and_null_context(built_lib):
    from rls_b200._lib import lib
    L = lib()
    assert L.rls_status_string(0) == b"ok"
    assert L.rls_status_string(-2) == b"dimension mismatch"
    assert L.rls_status_string(-5) == b"bounded device wait expired"
    assert L.rls_last_error(None)
    # grid entry points are pure host code and validate their arguments
    from rls_b200._lib import rls_grid
    g = rls_grid(0.0, 1.0, 0.0, 1.0, 1, 4, 1)
    assert L.rls_grid_zigzag(C.byref(g), None) == -1


def test_lanes_reject_a_context_listed_twice(built_lib):
    """Each lane's host thread drives its own context; a context listed twice is an
    ArgumentError found before any context is touched (the pointers here are never read)."""
    from rls_b200._lib import lib, rls_grid, rls_pstrirecy_control
    L = lib()
    fake = C.create_string_buffer(64)                     # stands in for one context handle
    ctxs = (C.c_void_p * 3)(C.addressof(fake), C.addressof(fake) + 16, C.addressof(fake))
    g = rls_grid(0.0, 1.0, 0.0, 1.0, 4, 4, 2)
    Z = (C.c_double * 32)()
    sig = (C.c_double * 16)()
    ctl = rls_pstrirecy_control()
    st = L.rls_pstrirecy_schur_lanes(ctxs, 3, Z, 16, C.byref(g), C.byref(ctl), None, sig, None)
    assert st == -1
    assert b"share one context" in L.rls_last_error(None)
