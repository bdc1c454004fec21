"""The C-ABI library loads without a GPU and exports every declared symbol."""
import os
import re
import subprocess
import tempfile

from conftest import REPO

HEADER = os.path.join(REPO, "include", "mblbm.h")


def declared_symbols():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(mb_[a-zA-Z0-9_]+)\s*\(", txt)))


def test_exports_every_declared_symbol(mb):
    lib = mb.load()
    names = declared_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python mirror binds exactly those
    assert sorted(mb.SIGNATURES) == names


def test_nm_lists_symbols(mb):
    out = subprocess.run(["nm", "-D", "--defined-only", mb.LIB_PATH], capture_output=True, text=True).stdout
    for n in declared_symbols():
        assert re.search(rf"\bT {n}\b", out), n


def test_version_and_errors(mb):
    lib = mb.load()
    assert lib.mb_version() == 1
    assert lib.mb_error_string(0) == b"ok"
    assert b"geometry" in lib.mb_error_string(-4)
    assert lib.mb_error_string(-99) == b"unknown error"


def test_struct_layouts_match_c(mb):
    """ctypes mirrors have the sizes the C compiler gives the header structs."""
    src = """#include <stdio.h>
#include "mblbm.h"
int main(void){printf("%zu %zu %zu %zu %zu\\n", sizeof(mb_layout), sizeof(mb_config), sizeof(mb_area),
 sizeof(mb_line), sizeof(mb_geometry));return 0;}"""
    d = tempfile.mkdtemp()
    c = os.path.join(d, "s.c")
    open(c, "w").write(src)
    exe = os.path.join(d, "s")
    subprocess.run(["gcc", "-I", os.path.dirname(HEADER), c, "-o", exe], check=True)
    sizes = [int(v) for v in subprocess.run([exe], capture_output=True, text=True).stdout.split()]
    import ctypes as C

    assert sizes == [C.sizeof(mb.Layout), C.sizeof(mb.Config), C.sizeof(mb.Area), C.sizeof(mb.Line),
                     C.sizeof(mb.Geometry)]


def test_context_calls_fail_cleanly_without_device(mb):
    """No CUDA device here: mb_create reports it instead of falling back."""
    import ctypes as C

    import torch

    if torch.cuda.is_available():
        return
    g = mb.config1_geometry()
    h = C.c_void_p()
    rc = mb.load().mb_create(C.byref(g), 1, C.byref(h))
    assert rc == -9 and not h.value
