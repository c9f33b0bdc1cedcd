"""The C-ABI library without a GPU: it loads, and it exports exactly the
entry points that include/akb.h declares (no compute call is made)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared_symbols():
    import glob
    text = "".join(open(f).read() for f in sorted(glob.glob(os.path.join(ROOT, "include", "*.h"))))
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(akb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "akb_model_create" in syms and "akb_solve_steps" in syms
    assert len(syms) >= 20


def test_library_exports_every_declared_symbol():
    from akantu_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        _lib.build()
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_python_signatures_cover_header():
    from akantu_b200 import _lib
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_abi_version_and_error_string():
    from akantu_b200 import _lib
    L = _lib.lib()
    assert L.akb_abi_version() == 1
    assert isinstance(L.akb_last_error(), bytes)


def test_null_arguments_are_rejected_without_gpu():
    """Argument validation happens before any device call."""
    from akantu_b200 import _abi, _lib
    L = _lib.lib()
    assert L.akb_model_create(None, 1, None, None, None, None) == _abi.AKB_ERR_INVALID_ARGUMENT
    assert L.akb_solve_steps(None, 3) == _abi.AKB_ERR_INVALID_ARGUMENT
    assert b"null" in L.akb_last_error()
