"""The ctypes mirrors of the C-ABI structs (prrtc_b200/_lib.py) agree with
include/prrtc_b200.h field by field: a small C program compiled with gcc
prints sizeof and every offsetof, and the ctypes layout must match.  Host
logic only; no GPU."""
from __future__ import annotations

import ctypes as C
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent

PAIRS = {
    "Robot": "prrtc_robot_t", "World": "prrtc_world_t", "Inputs": "prrtc_inputs_t",
    "Outputs": "prrtc_outputs_t", "Attrs": "prrtc_attrs_t", "PointCloud": "prrtc_point_cloud_t",
    "Tuning": "prrtc_tuning_t", "BatchInputs": "prrtc_batch_inputs_t",
}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_ctypes_structs_match_header(tmp_path):
    from prrtc_b200 import _lib

    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "prrtc_b200.h"', "int main(void) {"]
    for py, c in PAIRS.items():
        cls = getattr(_lib, py)
        lines.append(f'printf("{py} size %zu\\n", sizeof({c}));')
        for name, _ in cls._fields_:
            lines.append(f'printf("{py} {name} %zu\\n", offsetof({c}, {name}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    seen = {}
    for line in out:
        if line.strip():
            py, name, value = line.split()
            seen[(py, name)] = int(value)
    for py in PAIRS:
        cls = getattr(_lib, py)
        assert seen[(py, "size")] == C.sizeof(cls), py
        for name, _ in cls._fields_:
            assert seen[(py, name)] == getattr(cls, name).offset, (py, name)
