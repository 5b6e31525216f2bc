"""3-D static-gantry (StaticCT) geometry, frame sequences and projector classes.

Same rays, in the same order, as the reference
(tomography/staticct_projector_3d.py:8-539): frame-major, then active
source, then illuminated module, then pixel with the module's v index
fastest (pixel = iu * det_ny + iv).  Gantry -> image per frame is
M_f @ x + b_f.  The float32 products are the same torch operations on the
same shapes as the reference's; per-module pixel positions are computed once.
"""
from __future__ import annotations

import math
from typing import Optional

import torch

from .. import _native as N
from .ct_projector_3d_module import CTProjector3DModule

__all__ = ["build_circular_sequence", "build_helical_sequence", "build_static_3d_geometry", "StaticCTProjector3D",
           "staticct_ray_tiling",
           "build_uniform_static_3d_geometry", "UniformStaticCTProjector3D"]


def build_circular_sequence(n_frame, n_source, device: Optional[torch.device] = None):
    """Identity gantry transforms; frame i fires source i mod n_source."""
    if device is None:
        device = torch.device("cuda" if torch.cuda.is_available() else "cpu")
    M = torch.eye(3, dtype=torch.float32, device=device).unsqueeze(0).repeat(n_frame, 1, 1)
    b = torch.zeros((n_frame, 3), dtype=torch.float32, device=device)
    active = torch.zeros(n_frame, n_source, dtype=torch.bool, device=device)
    active[torch.arange(n_frame), torch.arange(n_frame) % n_source] = True
    return M, b, active


def build_helical_sequence(n_frame, n_source, helical_travel_per_rot, device: Optional[torch.device] = None):
    """As the circular sequence, plus a z translation of
    (i - (n_frame-1)/2) * travel/n_source per frame."""
    step = helical_travel_per_rot / n_source
    M = torch.eye(3, dtype=torch.float32).unsqueeze(0).repeat(n_frame, 1, 1)
    b = torch.zeros((n_frame, 3), dtype=torch.float32)
    b[:, 2] = torch.tensor([(i - (n_frame - 1) / 2.0) * step for i in range(n_frame)], dtype=torch.float32)
    active = torch.zeros(n_frame, n_source, dtype=torch.bool)
    active[torch.arange(n_frame), torch.arange(n_frame) % n_source] = True
    if device is not None:
        M, b, active = M.to(device), b.to(device), active.to(device)
    return M, b, active


def build_static_3d_geometry(source_positions, module_centers, module_orientations, det_nx_per_module,
                             det_ny_per_module, det_spacing_x, det_spacing_y, source_module_mask, M_gantry, b_gantry,
                             active_sources, device: Optional[torch.device] = None):
    if device is None:
        device = torch.device("cuda" if torch.cuda.is_available() else "cpu")
    mu, mv = (det_nx_per_module - 1) / 2.0, (det_ny_per_module - 1) / 2.0
    local = torch.tensor([[(iu - mu) * det_spacing_x, (iv - mv) * det_spacing_y, 0.0]
                          for iu in range(det_nx_per_module) for iv in range(det_ny_per_module)],
                         dtype=torch.float32)
    cpu = lambda t: t.detach().cpu()  # noqa: E731
    Mg, bg, sp, mc, mo = cpu(M_gantry), cpu(b_gantry), cpu(source_positions), cpu(module_centers), \
        cpu(module_orientations)
    active, mask = cpu(active_sources).tolist(), cpu(source_module_mask).tolist()
    n_frame, n_source, n_module = Mg.shape[0], sp.shape[0], mc.shape[0]
    pix_gantry = []
    for m in range(n_module):
        p = local @ mo[m].transpose(0, 1)
        p += mc[m]
        pix_gantry.append(p)
    srcs, dsts = [], []
    for f in range(n_frame):
        Mf, bf = Mg[f], bg[f]
        for s in range(n_source):
            if not active[f][s]:
                continue
            s_img = Mf @ sp[s] + bf
            for m in range(n_module):
                if not mask[s][m]:
                    continue
                p_img = pix_gantry[m] @ Mf.transpose(0, 1) + bf
                srcs.append(s_img.unsqueeze(0).expand_as(p_img))
                dsts.append(p_img)
    if not srcs:
        empty = torch.empty((0, 3), dtype=torch.float32, device=device)
        return empty, empty.clone()
    return torch.cat(srcs, dim=0).to(device), torch.cat(dsts, dim=0).to(device)


class StaticCTProjector3D(CTProjector3DModule):
    """Reference staticct_projector_3d.py:174-271."""

    def __init__(self, n_x, n_y, n_z, M_gantry, b_gantry, source_positions, module_centers, module_orientations,
                 det_nx_per_module, det_ny_per_module, det_spacing_x, det_spacing_y, source_module_mask,
                 active_sources, M, b, backend="cuda", device: Optional[torch.device] = None,
                 precomputed_intersections=False, tvals=None, use_compression=True, ray_tiling=None,
                 deterministic_adjoint=False):
        if device is None:
            device = torch.device("cuda" if torch.cuda.is_available() else "cpu")
        src, dst = build_static_3d_geometry(source_positions=source_positions, module_centers=module_centers,
                                            module_orientations=module_orientations,
                                            det_nx_per_module=det_nx_per_module,
                                            det_ny_per_module=det_ny_per_module, det_spacing_x=det_spacing_x,
                                            det_spacing_y=det_spacing_y, source_module_mask=source_module_mask,
                                            M_gantry=M_gantry, b_gantry=b_gantry, active_sources=active_sources,
                                            device=device)
        super().__init__(n_x=n_x, n_y=n_y, n_z=n_z, M=M.to(device), b=b.to(device), src=src, dst=dst,
                         backend=backend, device=device, precomputed_intersections=precomputed_intersections,
                         tvals=tvals, use_compression=use_compression, ray_tiling=ray_tiling,
                         deterministic_adjoint=deterministic_adjoint)
        self.M_gantry, self.b_gantry = M_gantry, b_gantry
        self.source_positions, self.module_centers, self.module_orientations = source_positions, module_centers, \
            module_orientations
        self.det_nx_per_module, self.det_ny_per_module = det_nx_per_module, det_ny_per_module
        self.det_spacing_x, self.det_spacing_y = det_spacing_x, det_spacing_y
        self.source_module_mask, self.active_sources = source_module_mask, active_sources


def build_uniform_static_3d_geometry(n_source, source_radius, source_z_offset, n_module, module_radius,
                                     module_z_offset, modules_per_source, device: Optional[torch.device] = None):
    """Source ring and inward-facing module ring; each source illuminates its
    `modules_per_source` farthest modules (reference :374-457)."""
    if device is None:
        device = torch.device("cuda" if torch.cuda.is_available() else "cpu")
    ang_s = torch.linspace(0, 2 * math.pi - 2 * math.pi / n_source, n_source, device=device).tolist()
    sp = torch.tensor([[source_radius * math.cos(a), source_radius * math.sin(a), source_z_offset] for a in ang_s],
                      dtype=torch.float32, device=device)
    ang_m = torch.linspace(0, 2 * math.pi - 2 * math.pi / n_module, n_module, device=device).tolist()
    up = torch.tensor([0.0, 0.0, 1.0], dtype=torch.float32, device=device)
    centres, rots = [], []
    for a in ang_m:
        cx, cy = module_radius * math.cos(a), module_radius * math.sin(a)
        centres.append([cx, cy, module_z_offset])
        nn = math.sqrt(cx * cx + cy * cy)
        nrm = (cx / nn, cy / nn, 0.0) if nn >= 1e-12 else (1.0, 0.0, 0.0)
        normal = torch.tensor(nrm, dtype=torch.float32, device=device)
        side = torch.linalg.cross(up, normal)
        if side.norm() < 1e-12:
            side = torch.tensor([1.0, 0.0, 0.0], dtype=torch.float32, device=device)
        side = side / side.norm()
        rots.append(torch.stack([side, torch.linalg.cross(normal, side), normal], dim=1))
    mc = torch.tensor(centres, dtype=torch.float32, device=device)
    mo = torch.stack(rots, dim=0)
    mask = torch.zeros((n_source, n_module), dtype=torch.bool, device=device)
    for i in range(n_source):
        far = torch.topk(torch.norm(mc - sp[i], dim=1), modules_per_source, largest=True).indices
        mask[i, far] = True
    return sp, mc, mo, mask


def staticct_ray_tiling(n_view, det_nx_per_module, det_ny_per_module, voxel_rule=1, block_threads=128):
    """Launch tiling for StaticCT rays ordered [view][column][row] per module
    (the order build_static_3d_geometry emits: for each active (frame,
    source, module) the module's columns, rows fastest), n_view = the number
    of (frame, source, module) triples.  The lanes of a warp run down module
    rows, which share one x-y line from the source: with 16 rows per column
    two 16-lane groups per warp take the column walk, with a multiple of 32
    rows whole warps do.  Other row counts get None (flat launch)."""
    if det_ny_per_module != 16 and det_ny_per_module % 32 != 0:
        return None
    rows = 16 if det_ny_per_module == 16 else 32
    per = det_nx_per_module * det_ny_per_module
    return N.tiling(n_view, det_ny_per_module, det_nx_per_module, per, 1, det_ny_per_module, tile_rows=rows,
                    block_threads=block_threads, voxel_rule=voxel_rule)


class UniformStaticCTProjector3D(StaticCTProjector3D):
    """Reference staticct_projector_3d.py:460-539."""

    def __init__(self, n_x, n_y, n_z, n_source, source_radius, source_z_offset, n_module, module_radius,
                 det_nx_per_module, det_ny_per_module, det_spacing_x, det_spacing_y, module_z_offset, M_gantry,
                 b_gantry, active_sources, modules_per_source, M, b, backend="cuda", precomputed_intersections=False,
                 tvals=None, use_compression=True, device: Optional[torch.device] = None, ray_tiling=None,
                 voxel_rule=0, deterministic_adjoint=False):
        """voxel_rule 0 is the reference's midpoint rule, 1 the crossing
        rule; either way the rays are tiled for the column walk
        (staticct_ray_tiling) unless a ray_tiling is given."""
        if device is None:
            device = torch.device("cuda" if backend == "cuda" and torch.cuda.is_available() else "cpu")
        if ray_tiling is None:
            n_view = int(torch.as_tensor(active_sources).sum()) * int(modules_per_source)
            ray_tiling = staticct_ray_tiling(n_view, det_nx_per_module, det_ny_per_module, voxel_rule=voxel_rule)
            if ray_tiling is None:
                ray_tiling = N.flat_opts(voxel_rule=voxel_rule, block_threads=128)
        sp, mc, mo, smm = build_uniform_static_3d_geometry(n_source=n_source, source_radius=source_radius,
                                                           source_z_offset=source_z_offset, n_module=n_module,
                                                           module_radius=module_radius,
                                                           module_z_offset=module_z_offset,
                                                           modules_per_source=modules_per_source, device=device)
        super().__init__(n_x=n_x, n_y=n_y, n_z=n_z, M_gantry=M_gantry.to(device), b_gantry=b_gantry.to(device),
                         source_positions=sp, module_centers=mc, module_orientations=mo,
                         det_nx_per_module=det_nx_per_module, det_ny_per_module=det_ny_per_module,
                         det_spacing_x=det_spacing_x, det_spacing_y=det_spacing_y, source_module_mask=smm,
                         active_sources=active_sources.to(device), M=M.to(device), b=b.to(device), backend=backend,
                         precomputed_intersections=precomputed_intersections, tvals=tvals,
                         use_compression=use_compression, device=device, ray_tiling=ray_tiling,
                         deterministic_adjoint=deterministic_adjoint)
