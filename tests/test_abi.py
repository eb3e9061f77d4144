"""The C ABI library loads and exports every entry point declared in include/pd_b200.h."""

import re
from pathlib import Path

from newton_solver_diff_phd_b200 import _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "pd_b200.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(pd_\w+)\(", text, flags=re.MULTILINE)))


def test_library_exports_every_declared_symbol():
    lib = _lib.library()
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)


def test_version_and_error_without_gpu():
    lib = _lib.library()
    assert b"sm_100a" in lib.pd_version()
    assert lib.pd_destroy(None) == 0
