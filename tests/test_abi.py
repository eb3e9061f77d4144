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


def test_struct_layouts_match_the_header(tmp_path):
    """Every ctypes mirror of a header struct has the C compiler's size and field offsets."""
    import ctypes
    import subprocess

    structs = {name: getattr(_lib, name) for name in ("PdMeshDesc", "PdOptions", "PdDiffPdOptions", "PdBatchOptions")}
    lines = ['#include <stddef.h>', '#include <stdio.h>', f'#include "{HEADER}"', "int main(void) {"]
    for name, mirror in structs.items():
        lines.append(f'  printf("{name} %zu\\n", sizeof({name}));')
        for field, _ in mirror._fields_:
            lines.append(f'  printf("{name}.{field} %zu\\n", offsetof({name}, {field}));')
    lines += ["  return 0;", "}"]
    source = tmp_path / "layout.c"
    source.write_text("\n".join(lines) + "\n")
    subprocess.run(["gcc", "-std=c11", str(source), "-o", str(tmp_path / "layout")], check=True)
    printed = dict(line.split() for line in subprocess.run([str(tmp_path / "layout")], check=True, capture_output=True,
                                                          text=True).stdout.splitlines())
    for name, mirror in structs.items():
        assert int(printed[name]) == ctypes.sizeof(mirror), name
        for field, _ in mirror._fields_:
            assert int(printed[f"{name}.{field}"]) == getattr(mirror, field).offset, f"{name}.{field}"
