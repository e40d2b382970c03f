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


def test_header_compiles_as_c99_and_links(tmp_path):
    """include/vlgpu.h is plain C: a C99 caller of the batch life cycle and of
    the asynchronous pipeline compiles without warnings and links against the
    library (nothing is run)."""
    src = tmp_path / "caller.c"
    src.write_text(r'''
#include <stdint.h>
#include "vlgpu.h"
int step(vlgpu_batch* b, const uint64_t* offs, const uint32_t* gids, const float* data,
         const vlgpu_cell_fields* fields, const double* dt, uint32_t* off, uint32_t* cnt,
         uint32_t* out_g, float* out_d, uint64_t cap) {
   uint64_t used = 0;
   int st = vlgpu_batch_upload_async(b, offs, gids, data);
   if (st == VLGPU_OK) st = vlgpu_accelerate(b, fields, dt, 0);
   if (st == VLGPU_OK) st = vlgpu_batch_download_begin(b);
   if (st == VLGPU_OK) st = vlgpu_batch_download_end(b, off, cnt, out_g, out_d, cap, &used);
   if (st == VLGPU_OK) st = vlgpu_batch_sync(b);
   return st;
}
int main(void) { return vlgpu_version() == 0; }
''')
    from vlasiator_b200.build import build
    build()
    lib_dir = os.path.dirname(vlgpu.LIB_PATH)
    exe = tmp_path / "caller"
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                        str(src), "-L", lib_dir, "-lvlgpu", "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_entry_points_reject_null_arguments():
    """Every status-returning entry point, given null pointers and zero sizes,
    returns VLGPU_EINVAL before it touches the device (so this runs without a
    GPU): the argument checks come first everywhere."""
    import ctypes
    lib = vlgpu.load()
    checked = 0
    for name, (res, args) in sorted(vlgpu.SIGNATURES.items()):
        if res is not ctypes.c_int:
            continue
        zeros = [0.0 if a in (ctypes.c_double, ctypes.c_float) else
                 None if (hasattr(a, "contents") or a in (ctypes.c_void_p, ctypes.c_char_p)) else 0 for a in args]
        assert getattr(lib, name)(*zeros) == 1, name  # VLGPU_EINVAL
        checked += 1
    assert checked >= 45
