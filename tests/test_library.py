"""The C-ABI library loads and exports every entry point include/amdk.h
declares (no GPU needed: nothing is called on a device)."""
import ctypes
import os
import re

from amdkiit_b200 import build

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "amdk.h")


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*(amdk_\w+)\s*\(", txt, re.M)))


def test_header_declares_entry_points():
    names = declared()
    assert "amdk_create" in names and "amdk_scf_iteration" in names and len(names) >= 20


def test_library_exports_every_symbol():
    lib = ctypes.CDLL(build.build())
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_built_for_sm100a():
    out = open(build.LIB, "rb").read()
    assert b"sm_100a" in out or b"sm_100" in out
