"""libspns.so loads and exports every symbol include/spns.h declares (no GPU needed)."""
import ctypes
import os
import re

import pytest

from spns_b200 import hit

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "spns.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(spns_[a-z0-9_]+)\s*\(", src)))


def test_header_lists_match_python_binding():
    assert set(declared_symbols()) == set(hit.EXPORTED_SYMBOLS)


def test_library_exports_every_declared_symbol():
    if not os.path.exists(hit.LIB_PATH):
        pytest.skip("libspns.so not built")
    lib = ctypes.CDLL(hit.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_status_strings():
    if not os.path.exists(hit.LIB_PATH):
        pytest.skip("libspns.so not built")
    L = hit.lib()
    assert L.spns_status_string(0) == b"ok"
    assert L.spns_status_string(-2) == b"unsupported size"
