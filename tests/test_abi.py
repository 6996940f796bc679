"""The C-ABI library loads and exports every entry point include/rt_api.h
declares (no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

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
    # RtMaterial: 17 scalars + 2×16 floats = 4*(1+3+3+1+1+1+3+1+1+1+1+1+1+1+16+16) bytes
    assert ctypes.sizeof(abi.RtMaterial) == 4 * (1 + 3 + 3 + 1 + 1 + 1 + 3 + 1 + 1 + 1 + 1 + 1 + 1 + 1 + 16 + 16)
    assert ctypes.sizeof(abi.RtHit) == 16
    assert ctypes.sizeof(abi.RtPassParams) == 4 * 11 + 4 + 8
