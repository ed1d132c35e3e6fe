"""The ctypes structures of the Python binding have the layouts that
include/replay.h gives its structs: every field's offset and every struct's
size, measured by a C program compiled against the header (no GPU)."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

from replay_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STRUCTS = {"rp_graph_info": _lib.GraphInfo, "rp_params": _lib.Params, "rp_sim_info": _lib.SimInfo,
           "rp_profile": _lib.Profile, "rp_tune_result": _lib.TuneResult}


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    d = tmp_path_factory.mktemp("abi")
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "replay.h"', "int main(void) {"]
    for name, cls in STRUCTS.items():
        lines.append(f'  printf("{name} size %zu\\n", sizeof({name}));')
        for field, _ in cls._fields_:
            lines.append(f'  printf("{name} {field} %zu\\n", offsetof({name}, {field}));')
    lines += ["  return 0;", "}"]
    src = d / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = d / "layout"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    table = {}
    for line in out.splitlines():
        name, field, value = line.split()
        table[(name, field)] = int(value)
    return table


@pytest.mark.parametrize("name", sorted(STRUCTS))
def test_ctypes_struct_matches_header(c_layout, name):
    cls = STRUCTS[name]
    assert C.sizeof(cls) == c_layout[(name, "size")], name
    for field, _ in cls._fields_:
        assert getattr(cls, field).offset == c_layout[(name, field)], (name, field)
