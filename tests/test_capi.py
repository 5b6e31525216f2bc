"""The C-ABI library loads, exports every function include/ctlab_b200.h
declares, and rejects bad arguments before touching the GPU.  CPU only: no
compute call is made."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "ctlab_b200.h")
LIB = os.path.join(ROOT, "ct_laboratory_b200", "_lib", "libctlab_b200.so")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ctlab_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared()
    assert "ctlab_forward_project_3d_on_the_fly" in names and len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(LIB)
    for name in declared():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (ctlab_\w+)", out))
    assert set(declared()) <= exported


def test_python_binding_covers_header():
    from ct_laboratory_b200 import _native
    assert set(declared()) <= set(_native.exported_symbols())
    assert _native.ABI_VERSION == 1


def test_validation_without_gpu():
    from ct_laboratory_b200 import _native as N
    lib = N.lib
    fake = ctypes.c_void_p(16)  # never dereferenced: validation fails first
    rc = lib.ctlab_forward_project_3d_on_the_fly(fake, 0, 4, 4, 4, fake, fake, 10, fake, fake, fake, None)
    assert rc == 1 and b"batch" in lib.ctlab_last_error()
    rc = lib.ctlab_forward_project_3d_on_the_fly(fake, 1, 0, 4, 4, fake, fake, 10, fake, fake, fake, None)
    assert rc == 1 and b"dimension" in lib.ctlab_last_error()
    rc = lib.ctlab_forward_project_3d_on_the_fly(fake, 1, 4, 4, 4, None, None, 10, fake, fake, fake, None)
    assert rc == 1 and b"src" in lib.ctlab_last_error()
    rc = lib.ctlab_compress_tvals_3d_ex(fake, 10, 5, fake, fake, ctypes.c_float(1.0), fake, fake, fake, 7, None)
    assert rc == 1 and b"mode" in lib.ctlab_last_error()
    rc = lib.ctlab_invert_matrix(fake, 4, fake, None, None)
    assert rc == 1
    t = N.tiling(2, 3, 4, 12, 4, 1, tile_rows=32, block_threads=256)
    rc = lib.ctlab_forward_project_3d_on_the_fly_ex(fake, 1, 4, 4, 4, fake, fake, 25, fake, fake, fake,
                                                    ctypes.byref(t), None)
    assert rc == 1 and b"tiling" in lib.ctlab_last_error()


def test_product_does_not_import_oracle():
    pkg = os.path.join(ROOT, "ct_laboratory_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h")):
                src = open(os.path.join(dirpath, f)).read()
                assert "oracle" not in src.replace("reference", ""), f
