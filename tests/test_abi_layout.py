"""The ctypes mirrors of the public structs (impact_b200/__init__.py) have the size and the field
offsets of the C definitions in include/impact_b200.h, as a C compiler lays them out.

A field added to one side only, or in a different place, would make the library read the Python
host's parameters shifted -- with no error -- so the layouts are compared field by field: a small
C program (compiled here with gcc against the header) prints sizeof and offsetof of every field.
"""
import ctypes as C
import json
import os
import shutil
import subprocess

import pytest

import impact_b200 as I

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# C struct name -> (ctypes mirror, C field names in the mirror's order)
STRUCTS = {
    "impact_b200_axis_tables": (I.AxisTables, [f for f, _ in I.AxisTables._fields_]),
    "impact_b200_case_desc": (I.CaseDesc, [f for f, _ in I.CaseDesc._fields_]),
    "impact_b200_coeffs": (I.Coeffs, [f for f, _ in I.Coeffs._fields_]),
    "impact_b200_solver_params": (I.SolverParams, [f for f, _ in I.SolverParams._fields_]),
    "impact_b200_solver_result": (I.SolverResult, [f for f, _ in I.SolverResult._fields_]),
    "impact_b200_step_params": (I.StepParams, [f for f, _ in I.StepParams._fields_]),
    "impact_b200_step_state": (I.StepState, [f for f, _ in I.StepState._fields_]),
}


def _c_layout(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "impact_b200.h"', "int main(void) {",
             '  printf("{");']
    first = True
    for name, (_, fields) in STRUCTS.items():
        sep = "" if first else ","
        first = False
        lines.append(f'  printf("{sep}\\"{name}\\": {{\\"size\\": %zu", sizeof({name}));')
        for f in fields:
            lines.append(f'  printf(", \\"{f}\\": %zu", offsetof({name}, {f}));')
        lines.append('  printf("}");')
    lines += ['  printf("}\\n");', "  return 0;", "}"]
    src = tmp_path / "layout.c"
    exe = tmp_path / "layout"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    return json.loads(subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout)


def test_ctypes_mirrors_match_the_c_header(tmp_path):
    c = _c_layout(tmp_path)
    for name, (mirror, fields) in STRUCTS.items():
        assert C.sizeof(mirror) == c[name]["size"], name
        for f in fields:
            assert getattr(mirror, f).offset == c[name][f], (name, f)
