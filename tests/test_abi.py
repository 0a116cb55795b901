"""The C-ABI libraries load and export every symbol include/*.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

from mbs_fast_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header: str) -> list[str]:
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(mbs_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


@pytest.mark.parametrize("header,lib", [("mbs_po_b200.h", "libmbs_po_b200.so"),
                                        ("mbs_mlp.h", "libmbs_po_b200.so"),
                                        ("mbs_host.h", "libmbs_host.so")])
def test_exports(header, lib):
    names = declared_functions(header)
    assert len(names) >= 5, names
    L = abi.load(lib)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, f"{lib} lacks {missing}"


def test_version_string():
    from mbs_fast_b200 import handler
    v = handler.lib().mbs_po_version().decode()
    assert "sm_100a" in v


def test_struct_sizes_match_header():
    # offsets of the ctypes mirrors follow the C declarations
    assert ctypes.sizeof(abi.Beams) == 4 + 4 + 8 + 8 + 13 * 8
    assert abi.Wave.legacy_sign.offset == 10 * 8
    assert ctypes.sizeof(abi.Grid) == 4 + 4 + 8 + 8 + 8


def test_library_missing_fails_loudly(tmp_path, monkeypatch):
    monkeypatch.setattr(abi, "LIB_DIR", str(tmp_path))
    monkeypatch.setattr(abi, "_LIBS", {})
    with pytest.raises(RuntimeError, match="missing"):
        abi.load("libmbs_po_b200.so")
