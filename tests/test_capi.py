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


def test_batch_plan_validation_without_gpu():
    from ct_laboratory_b200 import _native as N
    lib = N.lib
    assert lib.ctlab_batch_workspace_bytes(0) == -1 and lib.ctlab_batch_workspace_bytes(65536) == -1
    assert lib.ctlab_batch_workspace_bytes(4) >= 256 + 4 * 64
    fake = 256 * 1024  # never dereferenced: validation fails first
    scans = (N.Scan * 2)()
    for s in scans:
        s.ndim, s.n_ray, s.src, s.dst, s.M_inv, s.b = 2, 10, fake, fake, fake, fake
        s.image_in, s.sino_out = fake, fake
        s.dims[0], s.dims[1] = 8, 8
    plan = N.Batch()
    need = lib.ctlab_batch_workspace_bytes(2)
    rc = lib.ctlab_batch_plan(scans, 2, 256, ctypes.c_void_p(fake), need - 1, ctypes.byref(plan), None)
    assert rc == 1 and b"too small" in lib.ctlab_last_error()
    rc = lib.ctlab_batch_plan(scans, 2, 100, ctypes.c_void_p(fake), need, ctypes.byref(plan), None)
    assert rc == 1 and b"block_threads" in lib.ctlab_last_error()
    scans[1].ndim = 3
    rc = lib.ctlab_batch_plan(scans, 2, 256, ctypes.c_void_p(fake), need, ctypes.byref(plan), None)
    assert rc == 1 and b"ndim" in lib.ctlab_last_error()
    scans[1].ndim = 2
    scans[1].opts.voxel_rule = 1
    rc = lib.ctlab_batch_plan(scans, 2, 256, ctypes.c_void_p(fake), need, ctypes.byref(plan), None)
    assert rc == 1 and b"voxel_rule" in lib.ctlab_last_error()
    scans[1].opts.voxel_rule = 0
    scans[1].sino_out = None
    rc = lib.ctlab_batch_plan(scans, 2, 256, ctypes.c_void_p(fake), need, ctypes.byref(plan), None)
    assert rc == 1 and b"together" in lib.ctlab_last_error()
    rc = lib.ctlab_forward_project_batched(ctypes.byref(N.Batch()), 0, None)
    assert rc == 1 and b"plan" in lib.ctlab_last_error()


def test_product_does_not_import_oracle():
    pkg = os.path.join(ROOT, "ct_laboratory_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h")):
                src = open(os.path.join(dirpath, f)).read()
                assert "oracle" not in src.replace("reference", ""), f
