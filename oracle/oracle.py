"""CPU oracle for the Siddon projector — TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
and ``--impl reference`` legs may import this module.  It is the checker and
the CPU baseline; the product package ``ct_laboratory_b200`` never imports it.

This is a thin numpy/ctypes front end over ``oracle/_build/libsiddon_oracle.so``
(built from ``siddon_oracle.c`` by ``oracle/Makefile``).  Every routine
restates one piece of the reference ct_laboratory projector:

========================  =====================================================
routine                    reference it restates
========================  =====================================================
``isect_torch``            compute_intersections_{2d,3d}_torch
                           (tomography/ct_projector_3d_torch.py:78-158,
                           ct_projector_2d_torch.py:4-65)
``fwd_tvals_torch``        forward_project_{2d,3d}_torch (3d_torch.py:161-274)
``back_tvals_torch``       back_project_{2d,3d}_torch (3d_torch.py:277-386)
``fwd_otf_torch``          the reference CPU on-the-fly path: intersections +
``back_otf_torch``         tvals projector per ray chunk
                           (benchmark/projector_timing_benchmark.py:171-190)
``compress_torch``         compress_tvals_to_uint16 (3d_torch.py:4-65)
``decompress_torch``       decompress_tvals_from_uint16 (3d_torch.py:68-75)
``fwd/back_planesort``     ray_kernel_plane_sort (src/ct_projector_3d.cu:902-1012)
``fwd/back_dda2``          2-D on-the-fly kernels (src/ct_projector_2d.cu:246-413)
``compress_cuda``          compress_tvals_3d_kernel (ct_projector_3d.cu:160-212)
``fwd/back_comp_cuda``     compressed kernels (ct_projector_3d.cu:99-157,215-269)
========================  =====================================================

``dtype=np.float64`` selects the FP64 oracle (same code in double precision).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libsiddon_oracle.so")
_lib = None


def build() -> str:
    """Compile the oracle library with its Makefile (gcc, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def _stale() -> bool:
    if not os.path.exists(_LIB_PATH):
        return True
    t = os.path.getmtime(_LIB_PATH)
    return any(os.path.getmtime(os.path.join(_HERE, f)) > t
               for f in ("siddon_oracle.c", "siddon_oracle_impl.h", "Makefile"))


def _load():
    global _lib
    if _lib is None:
        if _stale():
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
    return _lib


def _sfx(dtype) -> str:
    return "_f64" if np.dtype(dtype) == np.float64 else "_f32"


def _arr(a, dtype):
    return np.ascontiguousarray(np.asarray(a, dtype=dtype))


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _dims(dims):
    d = np.ascontiguousarray(np.asarray(dims, dtype=np.int32))
    return d


def set_threads(n: int) -> None:
    _load().orc_set_threads(ctypes.c_int(int(n)))


def max_threads() -> int:
    return int(_load().orc_max_threads())


def minv(M, dtype=np.float32):
    """M^-1 in the given precision (the reference inverts M with torch.inverse)."""
    return _arr(np.linalg.inv(np.asarray(M, dtype=np.float64)), dtype)


def voxel_diag_len(M, dtype=np.float32) -> float:
    lib = _load()
    fn = getattr(lib, "orc_voxel_diag_len" + _sfx(dtype))
    fn.restype = ctypes.c_double if np.dtype(dtype) == np.float64 else ctypes.c_float
    return float(fn(_p(_arr(M, dtype))))


def isect_torch(dims, Mi, b, src, dst, dtype=np.float32):
    dims = _dims(dims)
    ndim = len(dims)
    Mi, b, src, dst = (_arr(x, dtype) for x in (Mi, b, src, dst))
    n_ray = src.shape[0]
    K = int(np.sum(dims + 1))
    out = np.empty((n_ray, K), dtype=dtype)
    getattr(_load(), "orc_isect_torch" + _sfx(dtype))(
        ctypes.c_int(ndim), _p(dims), _p(Mi), _p(b), _p(src), _p(dst), ctypes.c_int64(n_ray), _p(out))
    return out


def fwd_tvals_torch(img, tvals, Mi, b, src, dst, dtype=np.float32):
    img = _arr(img, dtype)
    dims = _dims(img.shape)
    tvals, Mi, b, src, dst = (_arr(x, dtype) for x in (tvals, Mi, b, src, dst))
    n_ray, K = tvals.shape
    out = np.empty(n_ray, dtype=dtype)
    getattr(_load(), "orc_fwd_tvals_torch" + _sfx(dtype))(
        ctypes.c_int(len(dims)), _p(dims), _p(img), _p(tvals), ctypes.c_int(K), _p(Mi), _p(b), _p(src), _p(dst),
        ctypes.c_int64(n_ray), _p(out))
    return out


def back_tvals_torch(sino, tvals, Mi, b, src, dst, dims, dtype=np.float32):
    dims = _dims(dims)
    sino, tvals, Mi, b, src, dst = (_arr(x, dtype) for x in (sino, tvals, Mi, b, src, dst))
    n_ray, K = tvals.shape
    out = np.zeros(tuple(int(d) for d in dims), dtype=dtype)
    getattr(_load(), "orc_back_tvals_torch" + _sfx(dtype))(
        ctypes.c_int(len(dims)), _p(dims), _p(sino), _p(tvals), ctypes.c_int(K), _p(Mi), _p(b), _p(src), _p(dst),
        ctypes.c_int64(n_ray), _p(out))
    return out


def fwd_otf_torch(img, Mi, b, src, dst, dtype=np.float32):
    img = _arr(img, dtype)
    dims = _dims(img.shape)
    Mi, b, src, dst = (_arr(x, dtype) for x in (Mi, b, src, dst))
    n_ray = src.shape[0]
    out = np.empty(n_ray, dtype=dtype)
    getattr(_load(), "orc_fwd_otf_torch" + _sfx(dtype))(
        ctypes.c_int(len(dims)), _p(dims), _p(img), _p(Mi), _p(b), _p(src), _p(dst), ctypes.c_int64(n_ray), _p(out))
    return out


def back_otf_torch(sino, Mi, b, src, dst, dims, dtype=np.float32):
    dims = _dims(dims)
    sino, Mi, b, src, dst = (_arr(x, dtype) for x in (sino, Mi, b, src, dst))
    out = np.zeros(tuple(int(d) for d in dims), dtype=dtype)
    getattr(_load(), "orc_back_otf_torch" + _sfx(dtype))(
        ctypes.c_int(len(dims)), _p(dims), _p(sino), _p(Mi), _p(b), _p(src), _p(dst), ctypes.c_int64(src.shape[0]),
        _p(out))
    return out


def compress_torch(tvals, src, dst, voxel_diag, scales=None, dtype=np.float32):
    tvals, src, dst = (_arr(x, dtype) for x in (tvals, src, dst))
    n_ray, K = tvals.shape
    u16 = np.empty((n_ray, K), dtype=np.uint16)
    starts = np.empty(n_ray, dtype=dtype)
    sc_out = np.empty(n_ray, dtype=dtype)
    sc_in = None if scales is None else _arr(scales, dtype)
    real = ctypes.c_double if np.dtype(dtype) == np.float64 else ctypes.c_float
    getattr(_load(), "orc_compress_torch" + _sfx(dtype))(
        _p(tvals), ctypes.c_int64(n_ray), ctypes.c_int(K), _p(src), _p(dst), real(voxel_diag),
        None if sc_in is None else _p(sc_in), _p(u16), _p(starts), _p(sc_out))
    return u16, starts, sc_out


def decompress_torch(u16, starts, scales, dtype=np.float32):
    u16 = np.ascontiguousarray(np.asarray(u16).view(np.uint16) if np.asarray(u16).dtype == np.int16 else u16,
                               dtype=np.uint16)
    starts, scales = _arr(starts, dtype), _arr(scales, dtype)
    n_ray, K = u16.shape
    out = np.empty((n_ray, K), dtype=dtype)
    getattr(_load(), "orc_decompress_torch" + _sfx(dtype))(
        _p(u16), _p(starts), _p(scales), ctypes.c_int64(n_ray), ctypes.c_int(K), _p(out))
    return out


def fwd_planesort(vol, Mi, b, src, dst, dtype=np.float32):
    vol = _arr(vol, dtype)
    dims = _dims(vol.shape)
    Mi, b, src, dst = (_arr(x, dtype) for x in (Mi, b, src, dst))
    out = np.empty(src.shape[0], dtype=dtype)
    getattr(_load(), "orc_fwd_planesort" + _sfx(dtype))(
        _p(dims), _p(vol), _p(Mi), _p(b), _p(src), _p(dst), ctypes.c_int64(src.shape[0]), _p(out))
    return out


def back_planesort(sino, Mi, b, src, dst, dims, dtype=np.float32):
    dims = _dims(dims)
    sino, Mi, b, src, dst = (_arr(x, dtype) for x in (sino, Mi, b, src, dst))
    out = np.zeros(tuple(int(d) for d in dims), dtype=dtype)
    getattr(_load(), "orc_back_planesort" + _sfx(dtype))(
        _p(dims), _p(sino), _p(Mi), _p(b), _p(src), _p(dst), ctypes.c_int64(src.shape[0]), _p(out))
    return out


def fwd_dda2(img, Mi, b, src, dst, dtype=np.float32):
    img = _arr(img, dtype)
    dims = _dims(img.shape)
    Mi, b, src, dst = (_arr(x, dtype) for x in (Mi, b, src, dst))
    out = np.empty(src.shape[0], dtype=dtype)
    getattr(_load(), "orc_fwd_dda2" + _sfx(dtype))(
        _p(dims), _p(img), _p(Mi), _p(b), _p(src), _p(dst), ctypes.c_int64(src.shape[0]), _p(out))
    return out


def back_dda2(sino, Mi, b, src, dst, dims, dtype=np.float32):
    dims = _dims(dims)
    sino, Mi, b, src, dst = (_arr(x, dtype) for x in (sino, Mi, b, src, dst))
    out = np.zeros(tuple(int(d) for d in dims), dtype=dtype)
    getattr(_load(), "orc_back_dda2" + _sfx(dtype))(
        _p(dims), _p(sino), _p(Mi), _p(b), _p(src), _p(dst), ctypes.c_int64(src.shape[0]), _p(out))
    return out


def compress_cuda(tvals, src, dst, voxel_diag, dtype=np.float32):
    tvals, src, dst = (_arr(x, dtype) for x in (tvals, src, dst))
    n_ray, K = tvals.shape
    u16 = np.empty((n_ray, K), dtype=np.uint16)
    starts = np.empty(n_ray, dtype=dtype)
    scales = np.empty(n_ray, dtype=dtype)
    real = ctypes.c_double if np.dtype(dtype) == np.float64 else ctypes.c_float
    getattr(_load(), "orc_compress_cuda" + _sfx(dtype))(
        _p(tvals), ctypes.c_int64(n_ray), ctypes.c_int(K), _p(src), _p(dst), real(voxel_diag), _p(u16),
        _p(starts), _p(scales))
    return u16, starts, scales


def fwd_comp_cuda(vol, u16, starts, scales, Mi, b, src, dst, dtype=np.float32):
    vol = _arr(vol, dtype)
    dims = _dims(vol.shape)
    u16 = np.ascontiguousarray(np.asarray(u16).view(np.uint16))
    starts, scales, Mi, b, src, dst = (_arr(x, dtype) for x in (starts, scales, Mi, b, src, dst))
    n_ray, K = u16.shape
    out = np.empty(n_ray, dtype=dtype)
    getattr(_load(), "orc_fwd_comp_cuda" + _sfx(dtype))(
        _p(dims), _p(vol), _p(u16), _p(starts), _p(scales), ctypes.c_int(K), _p(Mi), _p(b), _p(src), _p(dst),
        ctypes.c_int64(n_ray), _p(out))
    return out


def back_comp_cuda(sino, u16, starts, scales, Mi, b, src, dst, dims, dtype=np.float32):
    dims = _dims(dims)
    u16 = np.ascontiguousarray(np.asarray(u16).view(np.uint16))
    sino, starts, scales, Mi, b, src, dst = (_arr(x, dtype) for x in (sino, starts, scales, Mi, b, src, dst))
    n_ray, K = u16.shape
    out = np.zeros(tuple(int(d) for d in dims), dtype=dtype)
    getattr(_load(), "orc_back_comp_cuda" + _sfx(dtype))(
        _p(dims), _p(sino), _p(u16), _p(starts), _p(scales), ctypes.c_int(K), _p(Mi), _p(b), _p(src), _p(dst),
        ctypes.c_int64(n_ray), _p(out))
    return out


def count_segments(dims, Mi, b, src, dst, dtype=np.float32) -> int:
    dims = _dims(dims)
    Mi, b, src, dst = (_arr(x, dtype) for x in (Mi, b, src, dst))
    fn = getattr(_load(), "orc_count_segments" + _sfx(dtype))
    fn.restype = ctypes.c_int64
    return int(fn(ctypes.c_int(len(dims)), _p(dims), _p(Mi), _p(b), _p(src), _p(dst), ctypes.c_int64(src.shape[0])))
