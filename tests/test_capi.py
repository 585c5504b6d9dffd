"""The C-ABI library loads and exports every entry point include/*.h declares
(no GPU needed: nothing is called)."""
import ctypes
import os
import re

from nonstationary_mra_b200 import build, capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    inc = os.path.join(ROOT, "include")
    text = "".join(open(os.path.join(inc, f)).read() for f in sorted(os.listdir(inc)) if f.endswith(".h"))
    return sorted(set(re.findall(r"^\s*(?:mra_status|const char\*)\s+(mra_\w+)\s*\(", text, re.M)))


def test_header_declares_entry_points():
    names = declared()
    assert "mra_create" in names and "mra_loglik" in names and len(names) >= 10


def test_library_exports_every_declared_symbol():
    build.build()
    lib = ctypes.CDLL(capi.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert sorted(n for n, _, _ in capi.SIGNATURES) == declared()
