"""The C-ABI library loads and exports exactly what include/itr_gpu.h declares (CPU only:
no compute calls), and the context constructor fails cleanly without a GPU."""
from __future__ import annotations

import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "itr_gpu.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"\b(itr_gpu_[a-z_]+)\s*\(", src)))


def test_header_declares_the_boundary():
    syms = declared_symbols()
    for s in ("itr_gpu_create", "itr_gpu_destroy", "itr_gpu_run_batch", "itr_gpu_last_error", "itr_gpu_info"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    from itr_gpu import _lib
    lib = _lib.load()
    for s in declared_symbols():
        assert hasattr(lib, s), s
    assert set(declared_symbols()) == set(_lib.SIGNATURES), "ctypes table and header disagree"


def test_struct_layouts_match_header(tmp_path):
    """Compile the header with the C compiler and compare every struct's size and field
    offsets with the ctypes mirrors."""
    import subprocess
    from itr_gpu import _lib
    structs = {"itr_params": _lib.Params, "itr_grid": _lib.Grid, "itr_design": _lib.Design,
               "itr_objective": _lib.Objective, "itr_result": _lib.Result, "itr_group": _lib.Group,
               "itr_primitive": _lib.Primitive, "itr_design_space": _lib.DesignSpace, "itr_scene_view": _lib.SceneView}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from itr_gpu import DeviceError, GpuSolver
    with pytest.raises(DeviceError):
        GpuSolver()
