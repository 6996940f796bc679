"""The C-ABI library loads and exports every entry point include/rt_api.h
declares (no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"^\s*(?:int32_t|int64_t|void|float)\s+(rt_\w+)\s*\(", txt, re.M))
    return names


def test_library_exports_every_declared_symbol():
    from rustracer_b200.renderer import lib
    L = lib()
    syms = declared_symbols()
    assert {"rt_scene_create", "rt_render_pass", "rt_trace_closest"} <= syms
    missing = [s for s in sorted(syms) if not hasattr(L, s)]
    assert not missing, missing


def test_version_without_gpu():
    from rustracer_b200.renderer import lib
    assert lib().rt_version() == 1


def test_ctypes_struct_sizes_match_header_layout():
    from rustracer_b200 import abi
    # RtMaterial: 17 scalars + 2×16 floats + the PBR block (9 scalars, emission[3], strength) + 5 texture ids
    assert ctypes.sizeof(abi.RtMaterial) == 4 * (1 + 3 + 3 + 1 + 1 + 1 + 3 + 1 + 1 + 1 + 1 + 1 + 1 + 1 + 16 + 16 + 13 + 5)
    assert ctypes.sizeof(abi.RtHit) == 16
    assert ctypes.sizeof(abi.RtPassParams) == 4 * 11 + 4 + 8


def test_ctypes_layouts_match_the_c_compiler(tmp_path):
    """sizeof and field offsets of every ABI struct as gcc lays them out from
    include/rt_api.h, against the ctypes mirrors."""
    import shutil
    import subprocess
    from rustracer_b200 import abi
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    structs = {n: getattr(abi, n) for n in ("RtMaterial", "RtConvex", "RtShape", "RtTexture", "RtMedium",
                                             "RtBackground", "RtSceneDesc", "RtDevelopParams", "RtGuideParams",
                                             "RtCamera", "RtPassParams", "RtHit", "RtTuning", "RtPhotonEmitter",
                                             "RtPhotonParams", "RtBatchJob")}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "rt_api.h"', "int main(void) {"]
    for n, t in structs.items():
        lines.append(f'printf("{n} %zu\\n", sizeof({n}));')
        for f in t._fields_:
            lines.append(f'printf("{n}.{f[0]} %zu\\n", offsetof({n}, {f[0]}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", inc, str(src), "-o", str(exe)], check=True)
    out = dict(l.split() for l in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n") if l)
    for n, t in structs.items():
        assert int(out[n]) == ctypes.sizeof(t), n
        for f in t._fields_:
            assert int(out[f"{n}.{f[0]}"]) == getattr(t, f[0]).offset, f"{n}.{f[0]}"
