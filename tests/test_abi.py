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


@pytest.mark.parametrize("header", ["akb.h", "akb_fe2.h", "akb_mesh.h"])
@pytest.mark.parametrize("lang", [("gcc", "-std=c99", "c"), ("g++", "-std=c++11", "c++")],
                         ids=["c99", "c++11"])
def test_header_compiles_as_c_and_cpp(header, lang, tmp_path):
    """Each C-ABI header stands alone as pedantic C99 (what a cgo, JNI or
    ctypes binding parses) and C++11, without warnings."""
    import shutil
    import subprocess
    cc, std, xlang = lang
    if shutil.which(cc) is None:
        pytest.skip(cc + " not found")
    src = tmp_path / "use.c"
    src.write_text('#include "%s"\nint main(void) { return 0; }\n' % header)
    r = subprocess.run([cc, std, "-x", xlang, "-Wall", "-Wextra", "-pedantic", "-Werror",
                        "-fsyntax-only", "-I", os.path.join(ROOT, "include"), str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_integration_guide_matches_the_headers():
    """INTEGRATION.md names every entry point the headers declare, and no
    akb_ name the headers do not have (globs like akb_mlp_* aside)."""
    import glob
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    headers = "".join(open(f).read() for f in sorted(glob.glob(os.path.join(ROOT, "include",
                                                                          "*.h"))))
    in_headers = set(re.findall(r"\b(akb_[a-z0-9_]+)\b", headers))
    mentioned = {n for n in re.findall(r"\b(akb_[a-z0-9_]+)(?!\*)\b", doc)
                 if not n.endswith("_")}
    mentioned -= {"akb_fe2", "akb_mesh", "akb_msh", "akb_model"}  # file and type stems
    assert sorted(mentioned - in_headers) == []
    assert sorted(set(declared_symbols()) - mentioned) == []


@pytest.mark.parametrize("program", ["shim_plate.cc", "shim_fe2.cc", "shim_neumann.cc"])
def test_cpp_shim_programs_compile_without_warnings(program):
    """The header-only C++ shim and the programs written against it compile
    with -Wall -Wextra as errors (what a maintainer's build would use)."""
    import shutil
    import subprocess
    if shutil.which("g++") is None:
        pytest.skip("g++ not found")
    r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-fsyntax-only",
                        "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "cpp", program)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
