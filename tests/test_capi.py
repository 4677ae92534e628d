"""The C ABI library loads and exports every symbol include/vite_b200.h declares
(CPU only: no call that needs a GPU)."""
import ctypes
import os
import re

import vite_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "vite_b200.h")).read()
    return sorted(set(re.findall(r"\b(vg_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_the_python_list():
    assert sorted(vite_b200.EXPORTED_SYMBOLS) == declared_symbols()


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(vite_b200.library_path())
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_loads():
    L = vite_b200.lib()
    assert L.vg_last_error(None) == b"null context"
