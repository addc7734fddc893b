"""The C-ABI library loads and exports every symbol include/kerrsplat_b200.h declares (CPU only:
no compute call is made)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            names += re.findall(r"^\s*(?:int|const char\*|void)\s+(ks_\w+)\s*\(", src, flags=re.M)
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    for n in ("ks_context_create", "ks_regenerate", "ks_render", "ks_thin_image", "ks_march_samples"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from kerrsplat_b200 import _lib, build
    build.build(verbose=False)
    lib = ctypes.CDLL(_lib.LIB_PATH)
    for n in declared_symbols():
        assert hasattr(lib, n), n
    assert _lib.load() is not None
