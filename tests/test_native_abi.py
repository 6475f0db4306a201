"""CPU-side checks of the C ABI: the library loads and exports every function declared in
include/clothstep.h; on a machine without a usable device the product path fails loudly."""
import os
import re

import pytest

from clothsimulator_b200 import native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "clothstep.h")).read()
    return sorted(set(re.findall(r"^\s*(?:cs_status|const char\*)\s+(cs_\w+)\s*\(", text, re.M)))


def test_header_matches_binding_list():
    assert declared_functions() == sorted(native.EXPORTED)


def test_library_exports_every_declared_symbol():
    lib = native.load_library()
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_create_without_device_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(native.ClothStepError) as e:
        native.Context(0)
    assert e.value.status == native.CS_ERR_NO_DEVICE


def test_struct_layouts_match_header(tmp_path):
    """sizeof and member offsets of every ABI struct, compiled from the header with the host C
    compiler, against the ctypes / numpy layouts the binding passes."""
    import ctypes
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    structs = {
        "cs_material_desc": native.MaterialDesc, "cs_sheet_desc": native.SheetDesc,
        "cs_step_params": native.StepParams, "cs_step_stats": native.StepStats,
        "cs_detect_params": native.DetectParams, "cs_collision_params": native.CollisionParams,
        "cs_collision_stats": native.CollisionStats, "cs_tune_result": native.TuneResult,
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "clothstep.h"', "int main(void) {"]
    for cname, ct in structs.items():
        lines.append(f'printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for f, _ in ct._fields_:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append('printf("cs_proximity_desc sizeof %zu\\n", sizeof(cs_proximity_desc));')
    for f in native.PROXIMITY_DTYPE.names:
        lines.append(f'printf("cs_proximity_desc {f} %zu\\n", offsetof(cs_proximity_desc, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for ln in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        s, f, v = ln.split()
        got[(s, f)] = int(v)
    for cname, ct in structs.items():
        assert got[(cname, "sizeof")] == ctypes.sizeof(ct), cname
        for f, _ in ct._fields_:
            assert got[(cname, f)] == getattr(ct, f).offset, (cname, f)
    assert got[("cs_proximity_desc", "sizeof")] == native.PROXIMITY_DTYPE.itemsize
    for f in native.PROXIMITY_DTYPE.names:
        assert got[("cs_proximity_desc", f)] == native.PROXIMITY_DTYPE.fields[f][1], f
