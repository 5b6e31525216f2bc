"""Rolling-window multi-rotation projector (helical-like scans) on the B200
kernels.

Same class, constructor and results as the reference's MultiRotationProjector
(tomography/ct_projector_3d_multirot.py:13-393): rotation i projects the
z-window of ``n_z_window`` slices centred ``shift_offset`` slices further than
rotation i-1 (around ``scan_center_slice``, default the volume centre)
through ``base_projector``; slices outside the volume are padded by
``padding_mode``: "repeat" (nearest edge slice, without gradient through the
copies), "reflect" (mirrored about the edge voxel, zero beyond
``reflection_padding_slices`` if given) or anything else (zeros).
``forward(volume)`` returns [n_rays, n_rotations]; ``back_project(sino,
full_volume_z_size)`` returns [n_x, n_y, full_volume_z_size] by adding every
rotation's window adjoint into the slices it came from.

Where the reference projects the windows one rotation at a time, here all
rotations' windows go through the projector as one batch of volumes: one
forward launch and one adjoint launch for the whole scan when the base
projector is a projector module (``CTProjector3DModule`` or a
``RandomSubsetProjector`` over one).  With an ``OrderedSubsetProjector`` base
each subset's tables are loaded once and applied to the batch of all
rotations (the reference's subset-aware order).
"""
from __future__ import annotations

import torch
from torch import nn

from .ct_projector_3d_module import CTProjector3DModule
from .ct_projector_3d_subsets import OrderedSubsetProjector, RandomSubsetProjector

__all__ = ["MultiRotationProjector"]


def _reflect(idx, n):
    """Indices mirrored about the edge voxels into [0, n) (n >= 1)."""
    if n == 1:
        return torch.zeros_like(idx)
    period = 2 * n - 2
    m = torch.remainder(idx, period)
    return torch.where(m >= n, period - m, m)


class MultiRotationProjector(nn.Module):
    def __init__(self, base_projector, n_rotations, shift_offset, n_z_window, scan_center_slice=None,
                 padding_mode="repeat", reflection_padding_slices=None, verbose=False):
        super().__init__()
        self.base_projector = base_projector
        self.n_rotations = int(n_rotations)
        self.shift_offset = float(shift_offset)
        self.n_z_window = int(n_z_window)
        self.scan_center_slice = scan_center_slice
        self.padding_mode = padding_mode
        self.reflection_padding_slices = reflection_padding_slices
        self.verbose = verbose

    # -- geometry (reference :51-61) --------------------------------------------
    def _get_rotation_z_bounds(self, full_volume_z_size, rot_idx):
        if self.scan_center_slice is not None:
            center = float(self.scan_center_slice) - 0.5
        else:
            center = (full_volume_z_size - 1) / 2.0
        first = center - (self.n_rotations - 1) / 2.0 * self.shift_offset
        rot_center = first + rot_idx * self.shift_offset
        start = int(round(rot_center - (self.n_z_window - 1) / 2.0))
        return start, start + self.n_z_window

    def _window_index(self, z_size, start, end, device):
        """(source slice of every window slice, mask of slices that carry
        the volume) for one rotation under the padding mode."""
        idx = torch.arange(start, end, device=device)
        inside = (idx >= 0) & (idx < z_size)
        if self.padding_mode == "reflect":
            src = _reflect(idx, z_size)
            keep = torch.ones_like(inside)
            if self.reflection_padding_slices is not None:
                lim = self.reflection_padding_slices
                keep = (idx >= -lim) & (idx < z_size + lim)
            return src, keep
        if self.padding_mode == "repeat":
            return idx.clamp(0, z_size - 1), torch.ones_like(inside)
        return idx.clamp(0, z_size - 1), inside

    def _extract_volume_slice(self, full_volume, start_z, end_z):
        """The z-window [start_z, end_z) of the volume, padded per the mode
        (reference :63-152)."""
        z = full_volume.shape[-1]
        src, keep = self._window_index(z, start_z, end_z, full_volume.device)
        win = full_volume.index_select(-1, src)
        outside = (torch.arange(start_z, end_z, device=full_volume.device) < 0) | \
                  (torch.arange(start_z, end_z, device=full_volume.device) >= z)
        if self.padding_mode == "repeat" and bool(outside.any()):
            # padded copies of the edge slice carry values but no gradient
            win = torch.where(outside, win.detach(), win)
        if not bool(keep.all()):
            win = win * keep.to(win.dtype)
        return win.contiguous()

    def _windows(self, full_volume):
        z = full_volume.shape[-1]
        return torch.stack([self._extract_volume_slice(full_volume, *self._get_rotation_z_bounds(z, i))
                            for i in range(self.n_rotations)], dim=0)

    def _batchable(self):
        # these take a batch of volumes (and a batch of sinograms) in one call
        return isinstance(self.base_projector, (CTProjector3DModule, RandomSubsetProjector, OrderedSubsetProjector))

    # -- forward ------------------------------------------------------------------
    def forward(self, full_volume):
        """Forward-project -> [n_rays, n_rotations]."""
        if isinstance(full_volume, (list, tuple)):
            return [self.forward(v) for v in full_volume]
        if full_volume.dim() != 3:
            raise ValueError(f"MultiRotationProjector expects an [n_x, n_y, n_z] volume (got {tuple(full_volume.shape)})")
        windows = self._windows(full_volume.contiguous())  # [n_rot, n_x, n_y, n_z_window]
        bp = self.base_projector
        if self._batchable():
            return bp(windows).t().contiguous()
        return torch.stack([bp(windows[i]) for i in range(self.n_rotations)], dim=1).contiguous()

    # -- back-projection --------------------------------------------------------------
    def _scatter(self, shape, bp_windows, z_size):
        """Add every rotation's window adjoint into the slices it came from."""
        full_bp = torch.zeros((*shape, z_size), device=bp_windows.device, dtype=bp_windows.dtype)
        for i in range(self.n_rotations):
            start, end = self._get_rotation_z_bounds(z_size, i)
            src, keep = self._window_index(z_size, start, end, full_bp.device)
            w = bp_windows[i]
            if not bool(keep.all()):
                src, w = src[keep], w[..., keep]
            full_bp.index_add_(2, src, w)
        return full_bp

    def back_project(self, sino, full_volume_z_size):
        """sino [n_rays, n_rotations] -> [n_x, n_y, full_volume_z_size]."""
        bp = self.base_projector
        core = bp
        while hasattr(core, "base_projector") and not isinstance(core, CTProjector3DModule):
            core = core.base_projector
        shape = (core.n_x, core.n_y)
        sino_t = sino.t().contiguous()  # [n_rot, n_rays]: one row per rotation
        if self._batchable():
            wins = bp.back_project(sino_t)
            return self._scatter(shape, wins, int(full_volume_z_size))
        wins = torch.stack([bp.back_project(sino_t[i]) for i in range(self.n_rotations)], dim=0)
        return self._scatter(shape, wins, int(full_volume_z_size))
