"""The C-ABI library loads and exports every symbol include/*.h declares (no GPU needed)."""
import glob
import os
import re

import difftetvr_b200._lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


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
