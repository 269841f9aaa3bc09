"""The C-ABI library loads and exports every symbol include/*.h declares (no GPU needed)."""
import glob
import importlib.util
import os
import re

import difftetvr_b200._lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_cpp_build():
    """tests/cpp/build.py (compiles the C++ check program)."""
    spec = importlib.util.spec_from_file_location("cpp_check_build", os.path.join(ROOT, "tests", "cpp", "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(dtv_\w+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    lib = L.load()
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert declared_symbols() <= set(L.SIGNATURES), declared_symbols() - set(L.SIGNATURES)


def test_version_and_error_path():
    lib = L.load()
    assert lib.dtv_version() >= 100
    # Argument validation fails loudly without touching a GPU.
    code = lib.dtv_build_hex_mesh(None, None, 1, 1, 1, None, None)
    assert code == L.DTV_ERR_ARG
    assert b"null" in lib.dtv_last_error_string()


def test_cpp_classes_compile_against_the_headers_and_reject_bad_input():
    """include/difftetvr_b200.hpp (TetMesh / Renderer over the C ABI) compiles
    into a program linked to the in-tree library; its error paths that need
    no GPU throw difftetvr_b200::Error with the C ABI's codes."""
    import subprocess
    exe = load_cpp_build().build()
    res = subprocess.run([exe, "errors"], capture_output=True, text=True, timeout=60)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "OK errors" in res.stdout
