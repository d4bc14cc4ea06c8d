"""The ctypes mirrors of the C ABI's structs (spearhed_b200/abi.py) have the
layout the header declares (include/spearhed_b200.h): the same size and, for
every field, the same offset.  A small C program compiled with gcc against the
header prints sizeof and offsetof of each field; no CUDA call is made.

Array fields are compared by their first element's offset and the field's
total size, as ctypes reports them.
"""
import ctypes as C
import os
import subprocess

import pytest

from spearhed_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STRUCTS = ("SphParams", "SphBox", "SphSoAView", "SphDiag", "SphTuning", "SphLatticeBlock", "SphInitProfile")


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    d = tmp_path_factory.mktemp("layout")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "spearhed_b200.h"', 'int main(void) {']
    for name in STRUCTS:
        lines.append(f'  printf("{name} size %zu\\n", sizeof({name}));')
        for field, _ in getattr(abi, name)._fields_:
            lines.append(f'  printf("{name} {field} %zu %zu\\n", offsetof({name}, {field}), '
                         f'sizeof((({name}*)0)->{field}));')
    lines += ['  return 0;', '}']
    src = d / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = d / "layout"
    r = subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                        str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    layout = {}
    for line in out.splitlines():
        f = line.split()
        if f[1] == "size":
            layout[(f[0], None)] = (int(f[2]),)
        else:
            layout[(f[0], f[1])] = (int(f[2]), int(f[3]))
    return layout


@pytest.mark.parametrize("name", STRUCTS)
def test_ctypes_struct_matches_the_header(c_layout, name):
    S = getattr(abi, name)
    assert C.sizeof(S) == c_layout[(name, None)][0], name
    for field, _ in S._fields_:
        desc = getattr(S, field)
        assert (desc.offset, desc.size) == c_layout[(name, field)], (name, field)
