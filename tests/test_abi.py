"""The C-ABI library loads and exports every entry point its header declares
(no compute call: this runs without a GPU)."""
import ctypes
import os
import re

from asohf_b200 import api, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in ["asohf_gpu.h"]:
        txt = open(os.path.join(ROOT, "include", h)).read()
        names |= set(re.findall(r"^\s*(?:int|int64_t|const char \*)\s*\*?\s*(asohf_\w+)\s*\(", txt, re.M))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "asohf_halofind_particles" in names and "asohf_density" in names
    assert len(names) >= 18


def test_library_exports_every_declared_symbol():
    build.build()
    lib = ctypes.CDLL(api.lib_path())
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings():
    build.build()
    L = api.load()
    for code in range(9):
        assert L.asohf_strerror(code).decode()
