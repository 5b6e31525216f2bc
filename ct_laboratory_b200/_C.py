"""Drop-in for the reference's compiled module ``ct_laboratory._C``.

The reference binds 13 host wrappers with pybind11 (src/bindings.cpp:65-104);
each takes and returns torch tensors and expects ``M_inv`` already inverted.
This module exposes the same 13 names with the same argument order and
return shapes, implemented over the C ABI of libctlab_b200.so
(include/ctlab_b200.h).  Outputs are allocated here with torch on the
inputs' device and every launch goes to the current torch stream (the
reference launches on the legacy default stream).

Argument checks follow the reference's TORCH_CHECKs (e.g. "volume/tvals must
be CUDA", "volume shape!") and add dtype/contiguity checks the reference
leaves to its Python wrappers (ct_projector_3d_cuda.py:134-143); violations
raise RuntimeError.
"""
from __future__ import annotations

import torch

import weakref
from collections import OrderedDict

from . import _layout
from . import _native as N

# Active-tile lists of bare calls (no launch hint): keyed by the geometry
# tensors (weak references plus their versions: a freed tensor's address
# that comes back with other contents never matches) and by the values of
# M^-1 and b, which callers such as the reference's wrappers rebuild on
# every call.  Comparing those 12 values reads them to the host once per
# call.
_BARE_TILES = OrderedDict()
_BARE_TILES_MAX = 8


def _bare_active(tiling, src, dst, M_inv, b, dims):
    if tiling is None or tiling.n_view == 0:
        return tiling
    vals = torch.cat([M_inv.reshape(-1), b.reshape(-1)]).cpu()
    key = (id(src), id(dst), tuple(int(v) for v in dims), tuple(getattr(tiling, f) for f, _ in N.RayOpts._fields_))
    hit = _BARE_TILES.get(key)
    if (hit is not None and hit[0]() is src and hit[1]() is dst and hit[2] == (src._version, dst._version)
            and torch.equal(hit[3], vals)):
        _BARE_TILES.move_to_end(key)
        return hit[4]
    opts = N.active_tiling(tiling, src, dst, M_inv, b, dims)
    _BARE_TILES[key] = (weakref.ref(src), weakref.ref(dst), (src._version, dst._version), vals, opts)
    while len(_BARE_TILES) > _BARE_TILES_MAX:
        _BARE_TILES.popitem(last=False)
    return opts

__all__ = [
    "compute_intersections_2d", "forward_project_2d_cuda", "back_project_2d_cuda",
    "forward_project_2d_on_the_fly_cuda", "back_project_2d_on_the_fly_cuda",
    "compute_intersections_3d", "forward_project_3d_cuda", "back_project_3d_cuda", "compress_tvals_3d_cuda",
    "forward_project_3d_compressed_cuda", "back_project_3d_compressed_cuda",
    "forward_project_3d_on_the_fly_cuda", "back_project_3d_on_the_fly_cuda",
]


def _check_cuda(msg, *ts):
    if not all(t.is_cuda for t in ts):
        raise RuntimeError(msg)


def _f32c(name, t):
    if t.dtype != torch.float32:
        raise RuntimeError(f"{name} must be float32 (got {t.dtype})")
    if not t.is_contiguous():
        raise RuntimeError(f"{name} must be C-contiguous")


def _geom(src, dst, M_inv, b, ndim):
    for name, t in (("src", src), ("dst", dst), ("M_inv", M_inv), ("b", b)):
        _f32c(name, t)
    if src.dim() != 2 or src.shape[1] != ndim or dst.shape != src.shape:
        raise RuntimeError(f"src/dst must be [n_ray, {ndim}] (got {tuple(src.shape)}, {tuple(dst.shape)})")
    if M_inv.numel() != ndim * ndim or b.numel() != ndim:
        raise RuntimeError(f"M_inv must have {ndim * ndim} and b {ndim} elements")
    dev = src.device
    if any(t.device != dev for t in (dst, M_inv, b)):
        raise RuntimeError("all tensors must be on the same device")


def _vol_shape(volume, ndim):
    if volume.dim() == ndim:
        return 1, tuple(volume.shape)
    if volume.dim() == ndim + 1:
        return volume.shape[0], tuple(volume.shape[1:])
    raise RuntimeError("volume shape!" if ndim == 3 else "image shape!")


def _sino_shape(sino):
    if sino.dim() == 1:
        return 1, sino.shape[0]
    if sino.dim() == 2:
        return sino.shape[0], sino.shape[1]
    raise RuntimeError("sino shape!")


# --------------------------------------------------------------------------- 2-D
def compute_intersections_2d(n_row, n_col, src, dst, M_inv, b):
    """src/ct_projector_2d.cu:158-177 -> [n_ray, (n_row+1)+(n_col+1)] float32."""
    _check_cuda("src/dst must be CUDA", src, dst)
    _check_cuda("M_inv/b must be CUDA", M_inv, b)
    _geom(src, dst, M_inv, b, 2)
    n_ray = src.shape[0]
    out = torch.empty((n_ray, (n_row + 1) + (n_col + 1)), device=src.device, dtype=torch.float32)
    with torch.cuda.device(src.device):
        N.call("ctlab_compute_intersections_2d", n_row, n_col, N.ptr(src), N.ptr(dst), n_ray, N.ptr(M_inv),
               N.ptr(b), N.ptr(out), N.stream_of(src))
    return out


def forward_project_2d_cuda(img, tvals, src, dst, M_inv, b):
    """src/ct_projector_2d.cu:179-200 -> [batch, n_ray]."""
    _check_cuda("img/tvals must be CUDA", img, tvals)
    _f32c("image", img)
    _f32c("tvals", tvals)
    _geom(src, dst, M_inv, b, 2)
    batch, (n_row, n_col) = _vol_shape(img, 2)
    n_ray = src.shape[0]
    out = torch.empty((batch, n_ray), device=img.device, dtype=torch.float32)
    with torch.cuda.device(img.device):
        N.call("ctlab_forward_project_2d_tvals", N.ptr(img), batch, n_row, n_col, N.ptr(tvals), tvals.shape[1],
               N.ptr(src), N.ptr(dst), n_ray, N.ptr(M_inv), N.ptr(b), N.ptr(out), N.stream_of(img))
    return out


def back_project_2d_cuda(sino, tvals, src, dst, M_inv, b, n_row, n_col):
    """src/ct_projector_2d.cu:202-221 -> [batch, n_row, n_col]."""
    _check_cuda("sino/tvals must be CUDA", sino, tvals)
    _f32c("sinogram", sino)
    _f32c("tvals", tvals)
    _geom(src, dst, M_inv, b, 2)
    batch, n_ray = _sino_shape(sino)
    out = torch.empty((batch, n_row, n_col), device=sino.device, dtype=torch.float32)
    with torch.cuda.device(sino.device):
        N.call("ctlab_back_project_2d_tvals", N.ptr(sino), batch, n_ray, N.ptr(tvals), tvals.shape[1], N.ptr(src),
               N.ptr(dst), N.ptr(M_inv), N.ptr(b), n_row, n_col, N.ptr(out), 0, N.stream_of(sino))
    return out


def forward_project_2d_on_the_fly_cuda(img, src, dst, M_inv, b):
    """src/ct_projector_2d.cu:416-440 (incremental march) -> [batch, n_ray]."""
    _check_cuda("inputs must be CUDA tensors", img, src, dst)
    _f32c("image", img)
    _geom(src, dst, M_inv, b, 2)
    batch, (n_row, n_col) = _vol_shape(img, 2)
    n_ray = src.shape[0]
    out = torch.empty((batch, n_ray), device=img.device, dtype=torch.float32)
    with torch.cuda.device(img.device):
        N.call("ctlab_forward_project_2d_on_the_fly", N.ptr(img), batch, n_row, n_col, N.ptr(src), N.ptr(dst), n_ray,
               N.ptr(M_inv), N.ptr(b), N.ptr(out), N.stream_of(img))
    return out


def back_project_2d_on_the_fly_cuda(sino, src, dst, M_inv, b, n_row, n_col):
    """src/ct_projector_2d.cu:442-465 -> [batch, n_row, n_col]."""
    _check_cuda("inputs must be CUDA tensors", sino, src, dst)
    _f32c("sinogram", sino)
    _geom(src, dst, M_inv, b, 2)
    batch, n_ray = _sino_shape(sino)
    out = torch.empty((batch, n_row, n_col), device=sino.device, dtype=torch.float32)
    with torch.cuda.device(sino.device):
        N.call("ctlab_back_project_2d_on_the_fly", N.ptr(sino), batch, n_ray, N.ptr(src), N.ptr(dst), N.ptr(M_inv),
               N.ptr(b), n_row, n_col, N.ptr(out), 0, N.stream_of(sino))
    return out


# --------------------------------------------------------------------------- 3-D
def compute_intersections_3d(n_x, n_y, n_z, src, dst, M_inv, b):
    """src/ct_projector_3d.cu:381-401 -> [n_ray, (n_x+1)+(n_y+1)+(n_z+1)]."""
    _check_cuda("src/dst must be CUDA", src, dst)
    _check_cuda("M_inv,b must be CUDA", M_inv, b)
    _geom(src, dst, M_inv, b, 3)
    n_ray = src.shape[0]
    out = torch.empty((n_ray, (n_x + 1) + (n_y + 1) + (n_z + 1)), device=src.device, dtype=torch.float32)
    with torch.cuda.device(src.device):
        N.call("ctlab_compute_intersections_3d", n_x, n_y, n_z, N.ptr(src), N.ptr(dst), n_ray, N.ptr(M_inv), N.ptr(b),
               N.ptr(out), N.stream_of(src))
    return out


def forward_project_3d_cuda(volume, tvals, src, dst, M_inv, b):
    """src/ct_projector_3d.cu:403-433 -> [batch, n_ray]."""
    _check_cuda("volume/tvals must be CUDA", volume, tvals)
    _check_cuda("src/dst must be CUDA", src, dst)
    _check_cuda("M_inv,b must be CUDA", M_inv, b)
    _f32c("volume", volume)
    _f32c("tvals", tvals)
    _geom(src, dst, M_inv, b, 3)
    batch, (n_x, n_y, n_z) = _vol_shape(volume, 3)
    n_ray = src.shape[0]
    out = torch.empty((batch, n_ray), device=volume.device, dtype=torch.float32)
    with torch.cuda.device(volume.device):
        N.call("ctlab_forward_project_3d_tvals", N.ptr(volume), batch, n_x, n_y, n_z, N.ptr(tvals), tvals.shape[1],
               N.ptr(src), N.ptr(dst), n_ray, N.ptr(M_inv), N.ptr(b), N.ptr(out), N.stream_of(volume))
    return out


def back_project_3d_cuda(sino, tvals, src, dst, M_inv, b, n_x, n_y, n_z):
    """src/ct_projector_3d.cu:435-462 -> [batch, n_x, n_y, n_z]."""
    _check_cuda("sino/tvals must be CUDA", sino, tvals)
    _check_cuda("src/dst must be CUDA", src, dst)
    _check_cuda("M_inv,b must be CUDA", M_inv, b)
    _f32c("sinogram", sino)
    _f32c("tvals", tvals)
    _geom(src, dst, M_inv, b, 3)
    batch, n_ray = _sino_shape(sino)
    out = torch.empty((batch, n_x, n_y, n_z), device=sino.device, dtype=torch.float32)
    with torch.cuda.device(sino.device):
        N.call("ctlab_back_project_3d_tvals", N.ptr(sino), batch, n_ray, N.ptr(tvals), tvals.shape[1], N.ptr(src),
               N.ptr(dst), N.ptr(M_inv), N.ptr(b), n_x, n_y, n_z, N.ptr(out), 0, N.stream_of(sino))
    return out


def compress_tvals_3d_cuda(tvals, src, dst, voxel_diag_len):
    """src/ct_projector_3d.cu:464-489 -> (int16 [n_ray, n_int], start [n_ray], scale [n_ray])."""
    return compress_tvals_3d_mode(tvals, src, dst, voxel_diag_len, mode=0)


def compress_tvals_3d_mode(tvals, src, dst, voxel_diag_len, mode=0):
    """The compressor with an encoder choice: 0 = the reference CUDA kernel's,
    1 = the reference torch function's (compress_tvals_to_uint16)."""
    _check_cuda("Inputs must be CUDA", tvals, src, dst)
    _f32c("tvals", tvals)
    _f32c("src", src)
    _f32c("dst", dst)
    n_ray, n_int = tvals.shape
    t16 = torch.empty((n_ray, n_int), device=tvals.device, dtype=torch.int16)
    start = torch.empty((n_ray,), device=tvals.device, dtype=torch.float32)
    scale = torch.empty((n_ray,), device=tvals.device, dtype=torch.float32)
    with torch.cuda.device(tvals.device):
        N.call("ctlab_compress_tvals_3d_ex", N.ptr(tvals), n_ray, n_int, N.ptr(src), N.ptr(dst),
               float(voxel_diag_len), N.ptr(t16), N.ptr(start), N.ptr(scale), int(mode), N.stream_of(tvals))
    return t16, start, scale


def forward_project_3d_compressed_cuda(volume, t_uint16, t_start, t_scale, src, dst, M_inv, b):
    """src/ct_projector_3d.cu:491-522 -> [batch, n_ray]."""
    _check_cuda("Inputs must be CUDA", volume, t_uint16, t_start, t_scale)
    _f32c("volume", volume)
    _geom(src, dst, M_inv, b, 3)
    _check_table(t_uint16, t_start, t_scale, src.shape[0])
    batch, (n_x, n_y, n_z) = _vol_shape(volume, 3)
    n_ray = src.shape[0]
    out = torch.empty((batch, n_ray), device=volume.device, dtype=torch.float32)
    with torch.cuda.device(volume.device):
        N.call("ctlab_forward_project_3d_compressed", N.ptr(volume), batch, n_x, n_y, n_z, N.ptr(t_uint16),
               N.ptr(t_start), N.ptr(t_scale), t_uint16.shape[1], N.ptr(src), N.ptr(dst), n_ray, N.ptr(M_inv),
               N.ptr(b), N.ptr(out), N.stream_of(volume))
    return out


def back_project_3d_compressed_cuda(sino, t_uint16, t_start, t_scale, src, dst, M_inv, b, n_x, n_y, n_z):
    """src/ct_projector_3d.cu:524-553 -> [batch, n_x, n_y, n_z]."""
    _check_cuda("Inputs must be CUDA", sino, t_uint16, t_start, t_scale)
    _f32c("sinogram", sino)
    _geom(src, dst, M_inv, b, 3)
    batch, n_ray = _sino_shape(sino)
    _check_table(t_uint16, t_start, t_scale, n_ray)
    out = torch.empty((batch, n_x, n_y, n_z), device=sino.device, dtype=torch.float32)
    with torch.cuda.device(sino.device):
        N.call("ctlab_back_project_3d_compressed", N.ptr(sino), batch, n_ray, N.ptr(t_uint16), N.ptr(t_start),
               N.ptr(t_scale), t_uint16.shape[1], N.ptr(src), N.ptr(dst), N.ptr(M_inv), N.ptr(b), n_x, n_y, n_z,
               N.ptr(out), 0, N.stream_of(sino))
    return out


def forward_project_3d_on_the_fly_cuda(volume, src, dst, M_inv, b, tiling=None):
    """src/ct_projector_3d.cu:1018-1049 -> [batch, n_ray].  `tiling` (an
    _native.RayOpts) is an optional launch-shape hint, not in the reference;
    without one the detector layout of src / dst is detected once per
    geometry (_layout.detect_tiling), the reference's midpoint voxel rule is
    used, and only the tiles holding a ray that crosses the volume are
    launched (_bare_active: listed once per geometry)."""
    _check_cuda("inputs must be CUDA", volume, src, dst)
    _f32c("volume", volume)
    _geom(src, dst, M_inv, b, 3)
    batch, (n_x, n_y, n_z) = _vol_shape(volume, 3)
    if tiling is None:
        tiling = _bare_active(_layout.detect_tiling(src, dst), src, dst, M_inv, b, (n_x, n_y, n_z))
    n_ray = src.shape[0]
    out = torch.empty((batch, n_ray), device=volume.device, dtype=torch.float32)
    act = getattr(tiling, "active", None)  # a list of the active tiles (_native.active_tiling)
    with torch.cuda.device(volume.device):
        if act is not None:
            N.call("ctlab_forward_project_3d_on_the_fly_tiles", N.ptr(volume), batch, n_x, n_y, n_z, N.ptr(src),
                   N.ptr(dst), n_ray, N.ptr(M_inv), N.ptr(b), N.ptr(out), N.tiling_ref(tiling), N.ptr(act[0]),
                   act[1], N.stream_of(volume))
        else:
            N.call("ctlab_forward_project_3d_on_the_fly_ex", N.ptr(volume), batch, n_x, n_y, n_z, N.ptr(src),
                   N.ptr(dst), n_ray, N.ptr(M_inv), N.ptr(b), N.ptr(out), N.tiling_ref(tiling), N.stream_of(volume))
    return out


def back_project_3d_on_the_fly_cuda(sino, src, dst, M_inv, b, n_x, n_y, n_z, tiling=None):
    """src/ct_projector_3d.cu:1051-1079 -> [batch, n_x, n_y, n_z]; `tiling` as
    for the forward."""
    _check_cuda("inputs must be CUDA", sino, src, dst)
    _f32c("sinogram", sino)
    _geom(src, dst, M_inv, b, 3)
    if tiling is None:
        tiling = _bare_active(_layout.detect_tiling(src, dst), src, dst, M_inv, b, (n_x, n_y, n_z))
    batch, n_ray = _sino_shape(sino)
    out = torch.empty((batch, n_x, n_y, n_z), device=sino.device, dtype=torch.float32)
    act = getattr(tiling, "active", None)
    with torch.cuda.device(sino.device):
        if act is not None:
            N.call("ctlab_back_project_3d_on_the_fly_tiles", N.ptr(sino), batch, n_ray, N.ptr(src), N.ptr(dst),
                   N.ptr(M_inv), N.ptr(b), n_x, n_y, n_z, N.ptr(out), 0, N.tiling_ref(tiling), N.ptr(act[0]), act[1],
                   N.stream_of(sino))
        else:
            N.call("ctlab_back_project_3d_on_the_fly_ex", N.ptr(sino), batch, n_ray, N.ptr(src), N.ptr(dst),
                   N.ptr(M_inv), N.ptr(b), n_x, n_y, n_z, N.ptr(out), 0, N.tiling_ref(tiling), N.stream_of(sino))
    return out


def _check_table(t_uint16, t_start, t_scale, n_ray):
    if t_uint16.dtype not in (torch.int16, torch.uint16) or not t_uint16.is_contiguous():
        raise RuntimeError("t_uint16 must be a C-contiguous int16/uint16 tensor")
    _f32c("t_start", t_start)
    _f32c("t_scale", t_scale)
    if t_uint16.dim() != 2 or t_uint16.shape[0] != n_ray or t_start.numel() != n_ray or t_scale.numel() != n_ray:
        raise RuntimeError("compressed table must be [n_ray, n_int] with n_ray starts and scales")
