"""Seeded synthetic phantoms (the reference's benchmark data is not public:
its StaticCT geometry file and DICOM phantom are not in the repository, so
workloads use these instead).

ellipse_phantom_2d    water disk (0.019/mm) + random ellipses, values U(0, 0.02)/mm
ellipsoid_phantom_3d  random ellipsoids, values U(0, 0.02)/mm

Coordinates are world millimetres of a centred grid with the given pixel /
voxel size, matching standard_image_transform_{2d,3d}.
"""
from __future__ import annotations

import math

import torch

__all__ = ["ellipse_phantom_2d", "ellipsoid_phantom_3d"]


def ellipse_phantom_2d(n_row, n_col, pixel=1.0, n_ellipse=10, seed=0, device="cpu", water=0.019):
    g = torch.Generator().manual_seed(seed)
    r = (torch.arange(n_row, dtype=torch.float64) - (n_row - 1) / 2.0) * pixel
    c = (torch.arange(n_col, dtype=torch.float64) - (n_col - 1) / 2.0) * pixel
    X, Y = torch.meshgrid(r, c, indexing="ij")
    R = 0.45 * min(n_row, n_col) * pixel
    img = torch.where(X * X + Y * Y <= R * R, water, 0.0)
    for _ in range(n_ellipse):
        rad = R * 0.8 * math.sqrt(float(torch.rand(1, generator=g)))
        phi = 2 * math.pi * float(torch.rand(1, generator=g))
        cx, cy = rad * math.cos(phi), rad * math.sin(phi)
        a, b = [R * (0.05 + 0.25 * float(torch.rand(1, generator=g))) for _ in range(2)]
        th = math.pi * float(torch.rand(1, generator=g))
        val = 0.02 * float(torch.rand(1, generator=g))
        u = (X - cx) * math.cos(th) + (Y - cy) * math.sin(th)
        v = -(X - cx) * math.sin(th) + (Y - cy) * math.cos(th)
        img = torch.where((u / a) ** 2 + (v / b) ** 2 <= 1.0, torch.as_tensor(val, dtype=torch.float64), img)
    return img.to(torch.float32).to(device).contiguous()


def _rotation(g):
    q = torch.randn(4, generator=g, dtype=torch.float64)
    q = q / q.norm()
    w, x, y, z = q.tolist()
    return torch.tensor([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                         [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                         [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]], dtype=torch.float64)


def ellipsoid_phantom_3d(n_x, n_y, n_z, voxel=1.0, n_ellipsoid=12, seed=0, device="cpu"):
    g = torch.Generator().manual_seed(seed)
    dev = torch.device(device)
    axes = [((torch.arange(n, dtype=torch.float32, device=dev) - (n - 1) / 2.0) * voxel) for n in (n_x, n_y, n_z)]
    X, Y, Z = torch.meshgrid(*axes, indexing="ij")
    half = 0.5 * torch.tensor([n_x, n_y, n_z], dtype=torch.float64) * voxel
    vol = torch.zeros((n_x, n_y, n_z), dtype=torch.float32, device=dev)
    for _ in range(n_ellipsoid):
        centre = (torch.rand(3, generator=g, dtype=torch.float64) - 0.5) * half
        semi = half * (0.08 + 0.3 * torch.rand(3, generator=g, dtype=torch.float64))
        Rm = _rotation(g)
        val = 0.02 * float(torch.rand(1, generator=g))
        P = torch.stack([X - float(centre[0]), Y - float(centre[1]), Z - float(centre[2])], dim=-1)
        Q = P @ Rm.to(torch.float32).to(dev)
        inside = ((Q / semi.to(torch.float32).to(dev)) ** 2).sum(-1) <= 1.0
        vol = vol + inside.to(torch.float32) * val
        del P, Q, inside
    return vol.contiguous()
