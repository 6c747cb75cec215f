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


def test_reference_driver_binds_only_declared_entry_points():
    """The reference driver built against libspns resolves its solver calls to entry points of include/spns.h."""
    import subprocess
    exe = os.path.join(ROOT, "spns_b200", "dropin", "_build", "spns_hit_qa")
    if not os.path.exists(exe):
        pytest.skip("drop-in driver not built (needs the reference sources)")
    out = subprocess.run(["nm", "-D", "--undefined-only", exe], capture_output=True, text=True, check=True).stdout
    used = sorted(set(re.findall(r"\b(spns_[a-z0-9_]+)\b", out)))
    assert used, "driver does not call libspns"
    assert set(used) <= set(declared_symbols()), set(used) - set(declared_symbols())
    assert "spns_step" in used and "spns_create" in used
