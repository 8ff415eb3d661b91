"""The ctypes mirrors of the C-ABI structs (gbm3d_b200/_lib.py) against
include/gbm3d.h: a small C program compiled with the host compiler prints
sizeof and the offset of every field, which must equal ctypes' view.  A field
added to one side only (or in another order) fails here, on the CPU, instead
of corrupting arguments on the GPU."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

from gbm3d_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STRUCTS = [_lib.gbm3d_opts, _lib.gbm3d_filters, _lib.gbm3d_mixed_batch]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a host C compiler")
def test_ctypes_structs_match_header(tmp_path):
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "gbm3d.h"', "int main(void) {"]
    for st in STRUCTS:
        name = st.__name__
        lines.append(f'  printf("{name} sizeof %zu\\n", sizeof({name}));')
        for field, _ in st._fields_:
            lines.append(f'  printf("{name} {field} %zu\\n", offsetof({name}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for row in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        name, what, value = row.split()
        got[(name, what)] = int(value)
    for st in STRUCTS:
        name = st.__name__
        assert got[(name, "sizeof")] == C.sizeof(st), name
        for field, _ in st._fields_:
            assert got[(name, field)] == getattr(st, field).offset, f"{name}.{field}"
