"""The Python mirror of the C ABI structs (mercury_b200/_lib.py) against the
header: every field's offset and every struct's size, as a C compiler lays
them out (gcc on include/mercury_b200.h)."""
import ctypes
import os
import shutil
import subprocess

import pytest

from mercury_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STRUCTS = {
    "mb_environment": _lib.Environment,
    "mb_batch_desc": _lib.BatchDesc,
    "mb_launch_config": _lib.LaunchConfig,
    "mb_plan_stats": _lib.PlanStats,
}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_struct_layouts_match_the_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "mercury_b200.h"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    c = {}
    for line in out:
        if line:
            name, field, val = line.split()
            c[(name, field)] = int(val)
    for cname, py in STRUCTS.items():
        assert c[(cname, "size")] == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert c[(cname, f)] == getattr(py, f).offset, (cname, f)
