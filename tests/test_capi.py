"""The C-ABI library loads without a GPU and exports every symbol the public
header declares (no compute calls here)."""
import ctypes
import os
import re

from conftest import REPO


def header_symbols():
    txt = open(os.path.join(REPO, "include", "afr_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(afr_\w+)\s*\(", txt, re.M)))


def test_library_exports_every_declared_symbol():
    from autoflowcfd_b200 import _lib

    lib = ctypes.CDLL(_lib.LIB_PATH)
    syms = header_symbols()
    assert len(syms) >= 12
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(_lib.SIGNATURES)


def test_status_strings_and_version():
    from autoflowcfd_b200 import _lib

    assert _lib.LIB.afr_version() >= 100
    assert _lib.LIB.afr_status_string(0) == b"ok"
    assert _lib.LIB.afr_status_string(6) == b"index out of range"


def test_create_rejects_bad_order_without_touching_the_gpu():
    """Argument validation happens before any device call."""
    from autoflowcfd_b200 import _lib

    d = _lib.AfrMeshDesc()
    d.order = 7
    d.n_cells = 1
    d.n_faces = 1
    p = _lib.AfrParams()
    p.n_vars = 5
    h = ctypes.c_void_p()
    rc = _lib.LIB.afr_create(ctypes.byref(d), ctypes.byref(p), None, ctypes.byref(h))
    assert rc == _lib.AFR_EUNSUPPORTED and not h.value
