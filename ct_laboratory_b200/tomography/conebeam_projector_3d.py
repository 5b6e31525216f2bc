"""3-D cone-beam geometry and projector class.

``build_conebeam_3d_geometry`` (ct_laboratory_b200/ray_geometry.py) returns
the same rays as the reference's (tomography/conebeam_projector_3d.py:6-96),
ordered [view][det_v][det_u].

``ConeBeam3DProjector`` additionally passes the kernels a ray tiling with
rows = det_v and cols = det_u, so that the 32 lanes of a warp trace 32
vertically adjacent rays (the same x-y path, neighbouring k voxels).
"""
from __future__ import annotations

import torch

from .. import _native as N
from ..ray_geometry import build_conebeam_3d_geometry
from .ct_projector_3d_module import CTProjector3DModule
from .gather import panels_from_grid
from .standard_image_transform import standard_image_transform_3d

__all__ = ["build_conebeam_3d_geometry", "ConeBeam3DProjector", "conebeam_tiling"]


def conebeam_tiling(n_view, det_nx, det_ny, tile_rows=32, block_threads=128, voxel_rule=0, walk=0):
    """Launch tiling for rays ordered [view][det_v][det_u]: lanes along v.
    128 threads (32 rows x 4 columns) per CTA: a CTA's slot frees when its
    slowest warp finishes, and smaller CTAs lose less to that tail (measured
    3 % faster than 256 on the cone256 scan; 64 and 32 in between)."""
    return N.tiling(n_view, det_ny, det_nx, det_ny * det_nx, det_nx, 1, tile_rows=tile_rows,
                    block_threads=block_threads, voxel_rule=voxel_rule, walk=walk)


class ConeBeam3DProjector(CTProjector3DModule):
    """Cone-beam projector (reference conebeam_projector_3d.py:101-172)."""

    def __init__(self, n_x, n_y, n_z, n_view, det_nx, det_ny, sid, sdd, det_spacing=1.0, voxel_size=1.0,
                 angle_offset=0.0, backend="cuda", device=None, precomputed_intersections=False, tile_rows=32,
                 voxel_rule=0, deterministic_adjoint=False, walk=0, build_on_device=False, block_threads=128):
        if device is None:
            device = torch.device("cuda" if backend == "cuda" and torch.cuda.is_available() else "cpu")
        src, dst = build_conebeam_3d_geometry(n_view=n_view, det_nx=det_nx, det_ny=det_ny, sid=sid, sdd=sdd,
                                              det_spacing=det_spacing, angle_offset=angle_offset,
                                              volume_center_xyz=(0.0, 0.0, 0.0),
                                              device=device if build_on_device else None)
        M, b = standard_image_transform_3d(n_x=n_x, n_y=n_y, n_z=n_z, s_x=voxel_size, s_y=voxel_size,
                                           s_z=voxel_size)
        panels = None
        if deterministic_adjoint == "gather":
            panels = panels_from_grid(src, dst, [v * det_nx * det_ny for v in range(n_view)], det_nx, det_ny, 1,
                                      det_nx, device=device)
        super().__init__(n_x=n_x, n_y=n_y, n_z=n_z, M=M.to(device), b=b.to(device), src=src.to(device),
                         dst=dst.to(device), backend=backend, device=device,
                         precomputed_intersections=precomputed_intersections, panels=panels,
                         deterministic_adjoint=deterministic_adjoint,
                         ray_tiling=conebeam_tiling(n_view, det_nx, det_ny, tile_rows=tile_rows,
                                                    block_threads=block_threads, voxel_rule=voxel_rule, walk=walk))
        self.device = device
        self.n_view, self.det_nx, self.det_ny = n_view, det_nx, det_ny
        self.sid, self.sdd, self.det_spacing, self.voxel_size = sid, sdd, det_spacing, voxel_size
