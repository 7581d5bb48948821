"""libnsgpu.so loads and exports every entry point include/nsgpu.h declares
(no compute call: these run without a GPU)."""
import ctypes
import pathlib
import re

from neospice_b200 import _lib as L

HEADERS = sorted((pathlib.Path(__file__).resolve().parents[1] / "include").glob("*.h"))


def declared_functions():
    names = set()
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(nsg\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_loads():
    assert L.lib() is not None


def test_all_declared_symbols_exported():
    names = declared_functions()
    assert len(names) >= 12
    lib = ctypes.CDLL(str(L.LIB_PATH))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert declared_functions() <= set(L.SIGNATURES)


def test_last_error_after_misuse():
    lib = L.lib()
    assert lib.nsg_batch_solve(None, None, None) == L.NSG_ERR_INVALID
    assert b"null" in lib.nsg_last_error()


def test_negative_wait_limit_is_refused():
    lib = L.lib()
    assert lib.nsg_set_wait_limit(-1) == L.NSG_ERR_INVALID
    assert b"negative" in lib.nsg_last_error()
