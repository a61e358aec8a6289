"""The ctypes mirrors of the C ABI structs (ryoanji_b200/_abi.py) against the C header itself, on the host.

A small C program compiled with gcc prints sizeof and offsetof of every field the ctypes class declares; the
sizes and offsets must match field for field. A field missing or renamed on one side fails the compile.
"""
import ctypes as C
import os
import shutil
import subprocess

import pytest

from ryoanji_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PAIRS = {
    "ryo_box_f32": _abi.BoxF32,
    "ryo_box_f64": _abi.BoxF64,
    "ryo_group_view": _abi.GroupView,
    "ryo_ewald_settings": _abi.EwaldSettings,
    "ryo_traverse_options": _abi.TraverseOptions,
    "ryo_tree_view": _abi.TreeView,
    "ryo_solve_params": _abi.SolveParams,
    "ryo_solve_stats": _abi.SolveStats,
    "ryo_solve_arrays": _abi.SolveArrays,
    "ryo_system": _abi.System,
    "ryo_engine_params": _abi.EngineParams,
    "ryo_engine_request": _abi.EngineRequest,
    "ryo_engine_step_info": _abi.EngineStepInfo,
    "ryo_engine_result": _abi.EngineResult,
}


def _program():
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "ryoanji_b200.h"', "int main(void) {"]
    for cname, cls in PAIRS.items():
        lines.append(f'    printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for field, _ in cls._fields_:
            lines.append(f'    printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["    return 0;", "}"]
    return "\n".join(lines) + "\n"


def test_ctypes_structs_match_the_header(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "layout.c"
    src.write_text(_program())
    exe = tmp_path / "layout"
    r = subprocess.run([cc, "-std=c11", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    c = {}
    for line in out:
        if line:
            name, field, value = line.split()
            c[(name, field)] = int(value)
    for cname, cls in PAIRS.items():
        assert c[(cname, "sizeof")] == C.sizeof(cls), cname
        for field, _ in cls._fields_:
            assert c[(cname, field)] == getattr(cls, field).offset, (cname, field)
