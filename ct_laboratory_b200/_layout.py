"""Detector layout of a bare ray list, for the launch tiling of the 3-D
on-the-fly kernels.

The reference's compiled API (``_C.forward_project_3d_on_the_fly_cuda(volume,
src, dst, M_inv, b)``, src/bindings.cpp:98-101) receives rays without their
detector shape.  The column walk needs it: a warp's lanes must trace rays
that share one x-y line (one source, one detector column whose cells run
along z).  This module finds that structure in the ray list itself, once per
geometry, and returns the launch tiling for it.

Two orders are recognised, both as the reference's geometry builders emit
them:

* columns fastest, ``[view][row][column]`` (cone-beam, conebeam_projector_3d.py:
  84-94): ray r and ray r + n_col share the source and the detector cell's
  x and y;
* rows fastest, ``[view][column][row]`` (StaticCT modules,
  staticct_projector_3d.py:149-169): consecutive rays share them.

A view is the run of rays with the first ray's source.  The tiling is only a
launch hint: the kernels check per warp that the lanes really share their x-y
line and otherwise walk each ray on its own, so a layout that does not hold
everywhere costs time, never correctness.  Detection reads the first view and
a few sampled columns (a handful of small device-to-host copies) and is cached
per (src, dst) storage and version.
"""
from __future__ import annotations

from collections import OrderedDict

import torch

from . import _native as N

__all__ = ["detect_tiling", "clear_cache"]

_CACHE: "OrderedDict[tuple, object]" = OrderedDict()
_CACHE_MAX = 16
_FIRST_VIEW_MAX = 1 << 22  # rays searched for the end of the first view
_SAMPLES = 64              # columns checked across the scan


def clear_cache():
    _CACHE.clear()


def _key(src, dst, voxel_rule):
    return (src.data_ptr(), dst.data_ptr(), src._version, dst._version, src.shape[0], str(src.device),
            int(voxel_rule))


def _first_true(mask: torch.Tensor) -> int:
    """Index of the first True (mask.numel() when there is none)."""
    if mask.numel() == 0:
        return 0
    i = int(torch.argmax(mask.to(torch.uint8)))
    return i if bool(mask[i]) else mask.numel()


def _layout(src: torch.Tensor, dst: torch.Tensor):
    """(n_view, n_row, n_col, view_stride, row_stride, col_stride) or None."""
    n = src.shape[0]
    if n < 32:
        return None
    lim = min(n, _FIRST_VIEW_MAX)
    per_view = _first_true((src[:lim] != src[0]).any(dim=1))
    if (per_view == lim and lim < n) or n % per_view:
        return None  # a first view longer than the search, or views of unequal size
    xy = dst[:per_view, :2]
    same = (xy == xy[0]).all(dim=1)
    if per_view > 1 and bool(same[1]):
        # rows fastest: a column is the run of rays sharing the first x-y line
        n_row = _first_true(~same)
        if per_view % n_row:
            return None
        lay = (n // per_view, n_row, per_view // n_row, per_view, 1, n_row)
    else:
        k = _first_true(same[1:]) + 1
        if k >= per_view or per_view % k:
            return None
        lay = (n // per_view, per_view // k, k, per_view, k, 1)
    n_view, n_row, n_col, vs, rs, cs = lay
    if n_row < 16:
        return None
    # sampled columns of sampled views: every row shares the column's x-y
    # line and the view's source
    g = torch.Generator(device="cpu").manual_seed(n)
    v = torch.randint(0, n_view, (_SAMPLES,), generator=g)
    c = torch.randint(0, n_col, (_SAMPLES,), generator=g)
    idx = (v[:, None] * vs + c[:, None] * cs + torch.arange(n_row)[None, :] * rs).to(src.device)
    first = idx[:, :1]
    ok = (dst[idx, :2] == dst[first, :2]).all() & (src[idx] == src[first]).all()
    return lay if bool(ok) else None


def detect_tiling(src: torch.Tensor, dst: torch.Tensor, voxel_rule=N.VOXEL_MIDPOINT, block_threads=128):
    """Launch tiling (an _native.RayOpts) for a 3-D ray list, or None for the
    flat launch when no column layout is found."""
    key = _key(src, dst, voxel_rule)
    if key in _CACHE:
        _CACHE.move_to_end(key)
        return _CACHE[key]
    tiling = None
    lay = _layout(src, dst)
    if lay is not None:
        n_view, n_row, n_col, vs, rs, cs = lay
        rows = 32 if n_row % 32 == 0 else (16 if n_row == 16 else 0)
        if rows:
            tiling = N.tiling(n_view, n_row, n_col, vs, rs, cs, tile_rows=rows, block_threads=block_threads,
                              voxel_rule=voxel_rule)
    _CACHE[key] = tiling
    while len(_CACHE) > _CACHE_MAX:
        _CACHE.popitem(last=False)
    return tiling
