"""The C-ABI library loads on a host without a GPU and exports every entry
point include/vlgpu.h declares (no compute calls here)."""
import os
import re
import subprocess

from vlasiator_b200 import vlgpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"^\s*(?:int|const char\*)\s+(vlgpu_\w+)\s*\(", text, re.M))
    return names


def test_library_exports_all_declared_symbols():
    from vlasiator_b200.build import build
    build()
    lib = vlgpu.load()
    names = declared_symbols()
    assert len(names) >= 10
    for n in sorted(names):
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", vlgpu.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (vlgpu_\w+)", out))
    assert names <= exported, names - exported
    assert set(vlgpu.SIGNATURES) == names


def test_version_string():
    assert b"sm_100a" in vlgpu.load().vlgpu_version()
