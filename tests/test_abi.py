"""The C-ABI library loads on a machine without a GPU and exports every entry
point that include/vipe_b200.h declares (no compute calls are made here)."""

import re
from pathlib import Path

from vipe_b200 import _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "vipe_b200.h"


def _declared() -> set[str]:
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(vipe_\w+)\s*\(", text, flags=re.M))


def test_header_declares_the_bound_signatures():
    declared = _declared()
    assert len(declared) >= 39
    assert declared == set(_lib.EXPORTED)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    missing = [n for n in _declared() if getattr(lib, n, None) is None]
    assert not missing, missing
    assert _lib.missing_symbols() == []


def test_status_strings():
    assert _lib.status_string(0)
    assert "index" in _lib.status_string(_lib.VIPE_ERR_INDEX).lower()
