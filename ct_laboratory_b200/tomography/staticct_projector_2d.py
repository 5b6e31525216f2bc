"""2-D static-gantry (StaticCT) geometry and projector classes.

Same rays, in the same order, as the reference
(tomography/staticct_projector_2d.py:9-299): frame-major, then active
source, then illuminated module, then detector column.  A pixel's gantry
position is  R_m @ (offset, 0) + c_m  and every point is mapped to image
coordinates by the frame's  M_f @ x + b_f.  The matrix products are the same
torch operations on the same shapes as the reference's, so the float32
results agree exactly; the per-module pixel positions, which do not depend
on the frame, are computed once instead of once per (frame, source).
"""
from __future__ import annotations

import math
from typing import Optional

import torch

from .ct_projector_2d_module import CTProjector2DModule
from .gather import panels_from_lines_2d

__all__ = ["build_static_2d_geometry", "StaticCTProjector2D", "build_uniform_static_2d_geometry",
           "UniformStaticCTProjector2D"]


def build_static_2d_geometry(source_positions, module_center_positions, module_orientations, det_n_col, det_spacing,
                             source_module_mask, M_gantry, b_gantry, active_sources):
    device = source_positions.device
    n_frame, n_source, n_module = M_gantry.shape[0], source_positions.shape[0], module_center_positions.shape[0]
    mid = (det_n_col - 1) / 2.0
    local = torch.tensor([[(c - mid) * det_spacing, 0.0] for c in range(det_n_col)], dtype=torch.float32,
                         device=device)
    pix_gantry = [local @ module_orientations[m].transpose(0, 1) + module_center_positions[m] for m in range(n_module)]
    active = active_sources.cpu().tolist()
    mask = source_module_mask.cpu().tolist()
    srcs, dsts = [], []
    for f in range(n_frame):
        Mf, bf = M_gantry[f], b_gantry[f]
        for s in range(n_source):
            if not active[f][s]:
                continue
            s_img = Mf @ source_positions[s] + bf
            for m in range(n_module):
                if not mask[s][m]:
                    continue
                p_img = pix_gantry[m] @ Mf.transpose(0, 1) + bf
                srcs.append(s_img.unsqueeze(0).expand_as(p_img))
                dsts.append(p_img)
    if not srcs:
        empty = torch.empty((0, 2), dtype=torch.float32, device=device)
        return empty, empty.clone()
    return torch.cat(srcs, dim=0), torch.cat(dsts, dim=0)


class StaticCTProjector2D(CTProjector2DModule):
    """Reference staticct_projector_2d.py:92-149."""

    def __init__(self, n_row, n_col, M_gantry, b_gantry, source_positions, module_centers, module_orientations,
                 det_n_col, det_spacing, source_module_mask, active_sources, M, b, backend="cuda",
                 device: Optional[torch.device] = None, precomputed_intersections=False, deterministic_adjoint=False):
        src, dst = build_static_2d_geometry(source_positions=source_positions,
                                            module_center_positions=module_centers,
                                            module_orientations=module_orientations, det_n_col=det_n_col,
                                            det_spacing=det_spacing, source_module_mask=source_module_mask,
                                            M_gantry=M_gantry, b_gantry=b_gantry, active_sources=active_sources)
        if device is None:
            device = torch.device("cuda" if (backend == "cuda" and torch.cuda.is_available()) else "cpu")
        panels = None
        if deterministic_adjoint:  # one detector line per (frame, source, module)
            panels = panels_from_lines_2d(src, dst, list(range(0, src.shape[0], det_n_col)), det_n_col, 1,
                                          device=device)
        super().__init__(n_row=n_row, n_col=n_col, M=M.to(device), b=b.to(device), src=src.to(device),
                         dst=dst.to(device), backend=backend, precomputed_intersections=precomputed_intersections,
                         panels=panels, deterministic_adjoint=deterministic_adjoint)


def _ring_angles(n, device):
    return torch.linspace(0, 2 * math.pi - 2 * math.pi / n, n, device=device)


def build_uniform_static_2d_geometry(n_source, source_radius, n_module, module_radius, det_n_col, det_spacing,
                                     M_gantry, b_gantry, active_sources):
    """Sources and inward-facing modules on two rings; every source
    illuminates every module (reference staticct_projector_2d.py:155-216)."""
    device = M_gantry.device
    src_xy = [[source_radius * math.cos(a), source_radius * math.sin(a)] for a in
              _ring_angles(n_source, device).tolist()]
    centres, rots = [], []
    for a in _ring_angles(n_module, device).tolist():
        cx, cy = module_radius * math.cos(a), module_radius * math.sin(a)
        centres.append([cx, cy])
        nn = math.sqrt(cx * cx + cy * cy)
        nx, ny = (cx / nn, cy / nn) if nn >= 1e-12 else (1.0, 0.0)
        # columns: local x = in-plane tangent (-ny, nx), local y = normal
        rots.append(torch.tensor([[-ny, nx], [nx, ny]], dtype=torch.float32, device=device))
    return (torch.tensor(src_xy, dtype=torch.float32, device=device),
            torch.tensor(centres, dtype=torch.float32, device=device),
            torch.stack(rots, dim=0),
            torch.ones((n_source, n_module), dtype=torch.bool, device=device))


class UniformStaticCTProjector2D(StaticCTProjector2D):
    """Reference staticct_projector_2d.py:219-299."""

    def __init__(self, n_row, n_col, M, b, n_source, source_radius, n_module, module_radius, det_n_col, det_spacing,
                 M_gantry, b_gantry, active_sources, backend="cuda", device: Optional[torch.device] = None,
                 precomputed_intersections=False, deterministic_adjoint=False):
        if device is None:
            device = torch.device("cuda" if backend == "cuda" and torch.cuda.is_available() else "cpu")
        sp, mc, mo, smm = build_uniform_static_2d_geometry(n_source=n_source, source_radius=source_radius,
                                                           n_module=n_module, module_radius=module_radius,
                                                           det_n_col=det_n_col, det_spacing=det_spacing,
                                                           M_gantry=M_gantry, b_gantry=b_gantry,
                                                           active_sources=active_sources)
        super().__init__(n_row=n_row, n_col=n_col, M_gantry=M_gantry.to(device), b_gantry=b_gantry.to(device),
                         source_positions=sp.to(device), module_centers=mc.to(device),
                         module_orientations=mo.to(device), det_n_col=det_n_col, det_spacing=det_spacing,
                         source_module_mask=smm, active_sources=active_sources.to(device), M=M.to(device),
                         b=b.to(device), backend=backend, device=device,
                         precomputed_intersections=precomputed_intersections,
                         deterministic_adjoint=deterministic_adjoint)
        self.n_source, self.source_radius = n_source, source_radius
        self.n_module, self.module_radius = n_module, module_radius
        self.det_n_col, self.det_spacing = det_n_col, det_spacing
        self.device = device
