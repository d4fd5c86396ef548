"""The C ABI library loads on a machine without a GPU and exports every function that
include/mun_sem.h declares (no compute calls here)."""
import ctypes
import os
import re

from mun_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "mun_sem.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(sem_[a-z_]+)\s*\(",
                                 text, flags=re.M)))


def test_header_declares_the_entry_points():
    names = declared_functions()
    assert "sem_run" in names and "sem_plan_create" in names and len(names) >= 10


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    raw = ctypes.CDLL(lib._name)
    missing = [n for n in declared_functions() if not hasattr(raw, n)]
    assert not missing, missing
    assert set(_lib.EXPORTS) <= set(declared_functions())
