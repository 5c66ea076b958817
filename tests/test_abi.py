"""The C ABI: header declarations, the ctypes binding and the exported symbols agree (CPU)."""
import os
import re

import pytest

from dynlplus_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_functions():
    src = open(os.path.join(ROOT, "include", "dlp.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    out = {}
    for m in re.finditer(r"^\s*([A-Za-z_][\w\s\*]*?)\s*\b(dlp_\w+)\s*\(([^;]*?)\)\s*;", src, flags=re.M):
        ret, name, args = m.group(1).strip(), m.group(2), m.group(3).strip()
        codes = ""
        if args and args != "void":
            for a in args.split(","):
                a = " ".join(a.split())
                if "*" in a or a.startswith("dlp_stream_t"):
                    codes += "p"
                elif a.startswith(("int32_t", "int ")):
                    codes += "i"
                elif a.startswith("int64_t"):
                    codes += "q"
                elif a.startswith("double"):
                    codes += "d"
                elif a.startswith(("size_t", "unsigned long long")):
                    codes += "z"
                else:
                    raise AssertionError(f"unhandled parameter type in {name}: {a}")
        out[name] = (ret, codes)
    return out


def test_header_matches_binding():
    hdr = _header_functions()
    assert set(hdr) == set(_lib.SIGNATURES), set(hdr) ^ set(_lib.SIGNATURES)
    for name, (ret, codes) in hdr.items():
        assert _lib.SIGNATURES[name][0] == codes, (name, codes, _lib.SIGNATURES[name][0])


def test_library_exports_every_declared_symbol():
    if not os.path.exists(_lib.LIB_PATH):
        from dynlplus_b200 import build
        build.build()
    L = _lib.lib()
    for name in _header_functions():
        assert hasattr(L, name), name
    assert L.dlp_version() >= 1
    assert L.dlp_status_string(0) == b"ok"
    assert L.dlp_status_string(4) == b"iteration cap reached"


def test_argument_validation_without_device():
    """Shape errors are rejected on the host before any launch (no GPU needed)."""
    L = _lib.lib()
    # C = 0 is invalid
    st = L.dlp_spmm(None, None, None, None, 0, 10, None, 0, None, 1, 0, None, 1.0, 1.0, None, 1, 1.0, None, 1, 0,
                    0, 0, 0.0, None)
    assert st == 1
    # n_rows = 0 is a no-op
    st = L.dlp_spmm(None, None, None, None, 0, 0, None, 4, None, 4, 0, None, 1.0, 1.0, None, 4, 1.0, None, 4, 0, 0,
                    0, 0.0, None)
    assert st == 0
    # unsupported precision combination
    with pytest.raises(_lib.DLPError):
        _lib.call("dlp_spmm", 1, 1, 1, 1, 2, 4, None, 2, 16, 2, 0, None, 1.0, 1.0, None, 2, 1.0, 16, 2, 1, 0, 0,
                  0.0, None)
