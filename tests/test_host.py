"""CPU-only checks: the C-ABI library loads and exports every declared symbol."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "dendro_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(dg_[a-z0-9_]+)\s*\(", txt)))


def test_library_builds_and_exports_header_symbols():
    from dendro_b200 import build
    so = build.build()
    lib = ctypes.CDLL(so)
    syms = header_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_header():
    from dendro_b200 import _lib
    assert sorted(_lib.exported_symbols()) == header_symbols()


def test_no_device_reports_zero_or_more():
    from dendro_b200 import _lib
    assert _lib.lib().dg_device_count() >= 0


def test_status_strings():
    from dendro_b200 import _lib
    L = _lib.lib()
    for s in range(9):
        assert L.dg_status_string(s)
