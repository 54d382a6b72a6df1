"""The C-ABI library loads and exports every entry point include/cpstep.h declares."""
import os
import re

from openatom_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "cpstep.h")).read()
    return sorted(set(re.findall(r"CPSTEP_API\s+[\w\s\*]*?\b(cpstep_\w+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "cpstep_ctx_create" in names and "cpstep_density" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert missing == []


def test_python_binding_covers_header():
    assert sorted(_lib.SIGNATURES) == declared_symbols()


def test_version_and_error_text_without_gpu():
    L = _lib.lib()
    assert L.cpstep_version() >= 100
    assert isinstance(L.cpstep_last_error(), bytes)
