"""ctypes binding of libctlab_b200.so (the C ABI declared in include/ctlab_b200.h).

The library is required: importing this module raises ImportError when it
has not been built (``python ct_laboratory_b200/build.py``).  There is no
Python or CPU fallback for any projector.
"""
from __future__ import annotations

import ctypes
import os

import torch

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libctlab_b200.so")

if not os.path.exists(_LIB_PATH):
    raise ImportError(
        f"ct_laboratory_b200: native library {_LIB_PATH} is missing; build it with "
        "`python ct_laboratory_b200/build.py` (nvcc, sm_100a)")

lib = ctypes.CDLL(_LIB_PATH)

_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_I = ctypes.c_int
_F = ctypes.c_float


VOXEL_MIDPOINT = 0  # the reference's rule: rounded world-space segment midpoint
VOXEL_CROSSING = 1  # the voxel enclosed by the two bounding crossings (exact topology)
WALK_AUTO, WALK_LANE, WALK_COLUMN = 0, 1, 2


class RayOpts(ctypes.Structure):
    """Mirror of ctlab_ray_opts (include/ctlab_b200.h): ray tiling + voxel rule."""

    _fields_ = [("n_view", _I64), ("n_row", _I64), ("n_col", _I64), ("view_stride", _I64),
                ("row_stride", _I64), ("col_stride", _I64), ("tile_rows", ctypes.c_int32),
                ("block_threads", ctypes.c_int32), ("voxel_rule", ctypes.c_int32), ("walk", ctypes.c_int32)]


_TP = ctypes.POINTER(RayOpts)


class Scan(ctypes.Structure):
    """Mirror of ctlab_scan (include/ctlab_b200.h): one scan of a batch."""

    _fields_ = [("image_in", _P), ("sino_out", _P), ("sino_in", _P), ("image_out", _P), ("src", _P), ("dst", _P),
                ("M_inv", _P), ("b", _P), ("n_ray", _I64), ("dims", _I64 * 3), ("ndim", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("opts", RayOpts), ("image_scratch", _P)]


class Batch(ctypes.Structure):
    """Mirror of ctlab_batch (include/ctlab_b200.h): a plan of a batch."""

    _fields_ = [("workspace", _P), ("total_tiles", _I64), ("n_scan", ctypes.c_int32), ("ndim", ctypes.c_int32),
                ("block_threads", ctypes.c_int32), ("voxel_rule", ctypes.c_int32), ("has_forward", ctypes.c_int32),
                ("has_adjoint", ctypes.c_int32), ("device", ctypes.c_int32), ("has_scratch", ctypes.c_int32)]


_SP = ctypes.POINTER(Scan)
_BP = ctypes.POINTER(Batch)
_I32 = ctypes.c_int32

# name -> argtypes (every entry point returns int)
_SIGS = {
    "ctlab_forward_project_3d_on_the_fly": [_P, _I64, _I64, _I64, _I64, _P, _P, _I64, _P, _P, _P, _P],
    "ctlab_back_project_3d_on_the_fly": [_P, _I64, _I64, _P, _P, _P, _P, _I64, _I64, _I64, _P, _I, _P],
    "ctlab_forward_project_3d_on_the_fly_ex": [_P, _I64, _I64, _I64, _I64, _P, _P, _I64, _P, _P, _P, _TP, _P],
    "ctlab_back_project_3d_on_the_fly_ex": [_P, _I64, _I64, _P, _P, _P, _P, _I64, _I64, _I64, _P, _I, _TP, _P],
    "ctlab_compute_intersections_3d": [_I64, _I64, _I64, _P, _P, _I64, _P, _P, _P, _P],
    "ctlab_forward_project_3d_tvals": [_P, _I64, _I64, _I64, _I64, _P, _I64, _P, _P, _I64, _P, _P, _P, _P],
    "ctlab_back_project_3d_tvals": [_P, _I64, _I64, _P, _I64, _P, _P, _P, _P, _I64, _I64, _I64, _P, _I, _P],
    "ctlab_compress_tvals_3d": [_P, _I64, _I64, _P, _P, _F, _P, _P, _P, _P],
    "ctlab_compress_tvals_3d_ex": [_P, _I64, _I64, _P, _P, _F, _P, _P, _P, _I, _P],
    "ctlab_forward_project_3d_compressed": [_P, _I64, _I64, _I64, _I64, _P, _P, _P, _I64, _P, _P, _I64, _P, _P, _P,
                                            _P],
    "ctlab_back_project_3d_compressed": [_P, _I64, _I64, _P, _P, _P, _I64, _P, _P, _P, _P, _I64, _I64, _I64, _P, _I,
                                         _P],
    "ctlab_compute_intersections_2d": [_I64, _I64, _P, _P, _I64, _P, _P, _P, _P],
    "ctlab_forward_project_2d_tvals": [_P, _I64, _I64, _I64, _P, _I64, _P, _P, _I64, _P, _P, _P, _P],
    "ctlab_back_project_2d_tvals": [_P, _I64, _I64, _P, _I64, _P, _P, _P, _P, _I64, _I64, _P, _I, _P],
    "ctlab_forward_project_2d_on_the_fly": [_P, _I64, _I64, _I64, _P, _P, _I64, _P, _P, _P, _P],
    "ctlab_back_project_2d_on_the_fly": [_P, _I64, _I64, _P, _P, _P, _P, _I64, _I64, _P, _I, _P],
    "ctlab_forward_project_2d_siddon": [_P, _I64, _I64, _I64, _P, _P, _I64, _P, _P, _P, _TP, _P],
    "ctlab_back_project_2d_siddon": [_P, _I64, _I64, _P, _P, _P, _P, _I64, _I64, _P, _I, _TP, _P],
    "ctlab_back_project_2d_siddon_ws": [_P, _I64, _I64, _P, _P, _P, _P, _I64, _I64, _P, _I, _TP, _P, _P],
    "ctlab_invert_matrix": [_P, _I, _P, _P, _P],
    "ctlab_back_project_3d_gather": [_P, _I64, _I64, _P, _P, _P, _P, _P, _I64, _I64, _I64, _P, _I64, _P, _P],
    "ctlab_back_project_3d_gather_ws": [_P, _I64, _I64, _P, _P, _P, _P, _P, _I64, _I64, _I64, _P, _I64, _P, _P, _P],
    "ctlab_batch_plan": [_SP, _I32, _I32, _P, _I64, _BP, _P],
    "ctlab_forward_project_batched": [_BP, _I32, _P],
    "ctlab_back_project_batched": [_BP, _I, _I32, _P],
    "ctlab_batch_default_ctas": [_I32, _I, _I, _I32, ctypes.POINTER(_I32)],
    "ctlab_project_batched_noalloc": [_SP, _I32, _I, _I, _I32, _I32, _P],
    "ctlab_back_project_3d_fixed": [_P, _I64, _I64, _P, _P, _P, _P, _I64, _I64, _I64, _P, _I, _TP, _P, _I64, _P,
                                    _I64, _P],
    "ctlab_active_tiles": [_P, _P, _I64, _P, _P, _I64, _I64, _I64, _TP, _P, _P, _P, _P],
    "ctlab_forward_project_3d_on_the_fly_tiles": [_P, _I64, _I64, _I64, _I64, _P, _P, _I64, _P, _P, _P, _TP, _P,
                                                  _I64, _P],
    "ctlab_back_project_3d_on_the_fly_tiles": [_P, _I64, _I64, _P, _P, _P, _P, _I64, _I64, _I64, _P, _I, _TP, _P,
                                               _I64, _P],
    "ctlab_map_poisson_residual": [_P, _P, _P, _I64, _F, _P],
    "ctlab_map_smoothness_step": [_P, _P, _I64, _I64, _I64, _F, _F, _P],
}

for _name, _args in _SIGS.items():
    _fn = getattr(lib, _name)
    _fn.argtypes = _args
    _fn.restype = ctypes.c_int

lib.ctlab_last_error.restype = ctypes.c_char_p
lib.ctlab_last_error.argtypes = []
lib.ctlab_abi_version.restype = ctypes.c_int
lib.ctlab_abi_version.argtypes = []
lib.ctlab_batch_workspace_bytes.restype = ctypes.c_int64
lib.ctlab_batch_workspace_bytes.argtypes = [_I32]
lib.ctlab_tile_count.restype = ctypes.c_int64
lib.ctlab_tile_count.argtypes = [_I64, _TP]
lib.ctlab_back_project_3d_fixed_workspace_bytes.restype = ctypes.c_int64
lib.ctlab_back_project_3d_fixed_workspace_bytes.argtypes = [_I64, _I64, _I64, _I64]

ABI_VERSION = lib.ctlab_abi_version()


def exported_symbols():
    """Names of the C entry points this binding declares."""
    return sorted(_SIGS) + ["ctlab_last_error", "ctlab_abi_version", "ctlab_batch_workspace_bytes",
                            "ctlab_back_project_3d_fixed_workspace_bytes", "ctlab_tile_count"]


def call(name: str, *args) -> None:
    """Invoke an entry point and raise RuntimeError on a non-zero status."""
    rc = getattr(lib, name)(*args)
    if rc != 0:
        msg = lib.ctlab_last_error().decode(errors="replace")
        raise RuntimeError(f"{name} failed (status {rc}): {msg}")


def ptr(t):
    """Device pointer of a tensor (None -> NULL)."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def stream_of(t: torch.Tensor):
    """Raw handle of the current torch stream on t's device."""
    return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def tiling(n_view, n_row, n_col, view_stride, row_stride, col_stride, tile_rows=32, block_threads=256,
           voxel_rule=VOXEL_MIDPOINT, walk=WALK_AUTO):
    """Launch options for rays laid out as a [view][row][col] grid."""
    return RayOpts(int(n_view), int(n_row), int(n_col), int(view_stride), int(row_stride), int(col_stride),
                   int(tile_rows), int(block_threads), int(voxel_rule), int(walk))


def flat_opts(voxel_rule=VOXEL_MIDPOINT, block_threads=256):
    """Launch options for a flat ray list with a chosen voxel rule."""
    return RayOpts(0, 0, 0, 0, 0, 0, 0, int(block_threads), int(voxel_rule), WALK_AUTO)


def tiling_ref(t):
    return None if t is None else ctypes.byref(t)


class ActiveRayOpts(RayOpts):
    """RayOpts with the list of the tiling's active tiles (ctlab_active_tiles)
    as ``active = (int32 CUDA tensor, count)``: the on-the-fly 3-D calls of
    _C launch only those tiles (the *_tiles entry points)."""

    active = None


def active_tiling(t, src, dst, M_inv, b, dims):
    """An ActiveRayOpts copy of tiling `t` listing the tiles of the scan
    (src, dst, M_inv, b on one CUDA device; dims = (n_x, n_y, n_z)) that
    hold a ray the walks charge.  One pass over the rays and one host
    synchronisation (to read the count)."""
    n_ray = int(src.shape[0])
    n_blocks = int(lib.ctlab_tile_count(n_ray, ctypes.byref(t)))
    if n_blocks < 0:
        raise RuntimeError(f"ctlab_tile_count failed: {lib.ctlab_last_error().decode(errors='replace')}")
    dev = src.device
    flags = torch.empty(n_blocks, dtype=torch.uint8, device=dev)
    tiles = torch.empty(n_blocks, dtype=torch.int32, device=dev)
    count = torch.zeros(1, dtype=torch.int64, device=dev)
    with torch.cuda.device(dev):
        call("ctlab_active_tiles", ptr(src), ptr(dst), n_ray, ptr(M_inv), ptr(b), *[int(v) for v in dims],
             ctypes.byref(t), ptr(flags), ptr(tiles), ptr(count), stream_of(src))
    n = int(count.item())
    out = ActiveRayOpts()
    ctypes.memmove(ctypes.addressof(out), ctypes.addressof(t), ctypes.sizeof(RayOpts))  # copy the fields
    out.active = (tiles[:n].clone(), n)
    return out
