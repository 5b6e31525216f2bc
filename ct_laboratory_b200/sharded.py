"""One scan's rays split across GPUs: one process per GPU, torch.distributed.

The reference's multi-GPU projector (benchmark/multi_gpu_projector.py:59-144)
drives every GPU from a Python thread of one process, gives each a
contiguous shard of the rays with its own uint16 tables, and moves the
volume, the sinogram shards and the partial volumes between GPUs through
pinned host buffers.  Here every rank (one process per GPU) holds a
contiguous block of rays -- whole views when the projector has a detector
tiling, so that each rank keeps the column walk -- and projects it on the
fly (no tables to build).  The exchange is collective:

* forward: every rank projects its shard; ``gather_sinogram`` all-gathers
  the shards into the full sinogram on every rank (else each rank keeps its
  shard, ``local_sinogram``);
* adjoint: every rank back-projects its shard of the sinogram and the
  partial volumes are summed by one all-reduce;
* autograd: ``forward`` is differentiable, the backward being the sharded
  adjoint of the incoming gradient.

Every rank must make the same calls in the same order (they are collective).
"""
from __future__ import annotations

import math

import torch
import torch.distributed as dist
from torch import nn

from . import _native as N
from .tomography.ct_projector_3d_module import CTProjector3DModule

__all__ = ["RaySharded3DProjector", "shard_bounds"]


def shard_bounds(n_ray, world, align=1):
    """Contiguous ray ranges, one per rank, each a whole number of `align`
    rays (e.g. the rays of one view), the first ranks taking ceil shares as
    the reference's partition does (multi_gpu_projector.py:62-64)."""
    if n_ray % align:
        raise ValueError(f"n_ray ({n_ray}) is not a multiple of align ({align})")
    units = n_ray // align
    per = math.ceil(units / world) if units else 0
    out = []
    for r in range(world):
        lo, hi = min(r * per, units), min((r + 1) * per, units)
        out.append((lo * align, hi * align))
    return out


def _slice_module(m, lo, hi):
    """A CTProjector3DModule over rays [lo, hi) of module m, with its tables
    and its detector tiling (whole views) when it has them."""
    tiling = None
    t = m.ray_tiling
    if t is not None and t.n_view > 0:
        per_view = t.view_stride
        if lo % per_view or hi % per_view:
            raise ValueError("a tiled projector must be split at view boundaries")
        tiling = N.tiling((hi - lo) // per_view, t.n_row, t.n_col, t.view_stride, t.row_stride, t.col_stride,
                          tile_rows=t.tile_rows, block_threads=t.block_threads, voxel_rule=t.voxel_rule, walk=t.walk)
    tv = None
    if m.tvals_uint16 is not None:
        tv = (m.tvals_uint16[lo:hi], m.tvals_start[lo:hi], m.tvals_scale[lo:hi])
    elif m.tvals_full is not None:
        tv = m.tvals_full[lo:hi]
    # the fixed-point adjoint carries over to a slice; the gather needs the
    # whole scan's panel table, so a slice of a gathering module scatters
    fixed = getattr(m, "adjoint_mode", "atomic") == "fixed"
    return CTProjector3DModule(m.n_x, m.n_y, m.n_z, m.M, m.b, m.src[lo:hi], m.dst[lo:hi], backend=m.backend,
                               device=m.src.device, tvals=tv, use_compression=m.use_compression, ray_tiling=tiling,
                               deterministic_adjoint="fixed" if fixed else False)


class _Sharded(torch.autograd.Function):
    @staticmethod
    def forward(ctx, volume, proj):
        ctx.proj = proj
        with torch.no_grad():
            return proj.forward_project(volume)

    @staticmethod
    def backward(ctx, grad):
        return ctx.proj.back_project(grad.contiguous()), None


class RaySharded3DProjector(nn.Module):
    """`base` is a CTProjector3DModule holding the whole scan (every rank
    builds the same one, or loads it) or a factory ``(lo, hi) -> projector``
    for rays [lo, hi) together with ``n_ray``."""

    def __init__(self, base, n_ray=None, group=None, gather_sinogram=True, align=None):
        super().__init__()
        if not dist.is_initialized():
            raise RuntimeError("RaySharded3DProjector needs an initialised torch.distributed process group")
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.gather_sinogram = bool(gather_sinogram)
        if isinstance(base, CTProjector3DModule):
            n_ray = int(base.src.shape[0])
            if align is None:
                t = base.ray_tiling
                align = int(t.view_stride) if (t is not None and t.n_view > 0) else 1
            self.bounds = shard_bounds(n_ray, self.world, align)
            lo, hi = self.bounds[self.rank]
            self.local = _slice_module(base, lo, hi)
            self.n_x, self.n_y, self.n_z = base.n_x, base.n_y, base.n_z
        else:
            if n_ray is None:
                raise ValueError("a projector factory needs n_ray")
            self.bounds = shard_bounds(int(n_ray), self.world, align or 1)
            lo, hi = self.bounds[self.rank]
            self.local = base(lo, hi)
            self.n_x, self.n_y, self.n_z = (getattr(self.local, k, None) for k in ("n_x", "n_y", "n_z"))
        self.n_ray = int(n_ray)
        self.lo, self.hi = self.bounds[self.rank]
        self._max_shard = max(h - l for l, h in self.bounds)

    # -- collectives -----------------------------------------------------------
    def _gather(self, part):
        """All shards of the sinogram, in ray order, on every rank: one
        all_gather_into_tensor into a [world, ..., shard] buffer.  Shards may
        differ in length: each is then padded to the longest for the gather
        and the padding cut out after.  With equal shards and a single
        sinogram the buffer is the ray-ordered sinogram itself (no copy)."""
        lead = tuple(part.shape[:-1])
        m = self._max_shard
        equal = all(h - l == m for l, h in self.bounds)
        src = part.contiguous() if equal else part.new_zeros((*lead, m))
        if not equal:
            src[..., :part.shape[-1]] = part
        rows = int(torch.Size(lead).numel())
        buf = part.new_empty(self.world * rows * m)  # flat: every backend concatenates along dim 0
        dist.all_gather_into_tensor(buf, src.reshape(-1), group=self.group)
        if equal and rows == 1:
            return buf.reshape(*lead, self.world * m)
        buf = buf.reshape(self.world, rows, m)
        if equal:
            return buf.permute(1, 0, 2).reshape(*lead, self.world * m)
        return torch.cat([buf[r, :, :h - l] for r, (l, h) in enumerate(self.bounds)], dim=-1).reshape(*lead, -1)

    # -- projector API ------------------------------------------------------------
    def local_sinogram(self, volume):
        """This rank's shard of A volume (rays [lo, hi)), no communication."""
        return self.local.forward_project(volume)

    def forward_project(self, volume):
        part = self.local.forward_project(volume)
        return self._gather(part) if self.gather_sinogram else part

    def back_project(self, sinogram):
        """A^T sinogram on every rank: the full sinogram (or this rank's
        shard, when its length is the shard's) back-projected shard by shard
        and summed over the ranks."""
        if sinogram.shape[-1] == self.n_ray:
            sinogram = sinogram[..., self.lo:self.hi]
        elif sinogram.shape[-1] != self.hi - self.lo:
            raise ValueError(f"sinogram has {sinogram.shape[-1]} rays; expected {self.n_ray} or this rank's "
                             f"{self.hi - self.lo}")
        vol = self.local.back_project(sinogram.contiguous())
        dist.all_reduce(vol, op=dist.ReduceOp.SUM, group=self.group)
        return vol

    def forward(self, volume):
        if not self.gather_sinogram:
            raise RuntimeError("the differentiable forward returns the full sinogram: use gather_sinogram=True")
        return _Sharded.apply(volume, self)
