"""Named benchmark workloads (synthetic data with the configurations' shapes).

cone256  3-D cone-beam: 256^3 volume, 0.5 mm voxels; 360 views over 360
         degrees on a circular orbit; 512 x 384 detector at 0.8 mm;
         SID 1000 mm, SDD 1500 mm; 12 seeded ellipsoids, 0-0.02/mm.
         70,778,880 rays ordered [view][det_v][det_u].
fan256   2-D fan-beam: 256^2 image, 1 mm pixels; 360 views; 512 bins at
         1 mm; SID 1000 mm, SDD 1500 mm; water disk + 10 seeded ellipses.
         184,320 rays ordered [view][bin].
"""
from __future__ import annotations

from dataclasses import dataclass

__all__ = ["ConeWorkload", "FanWorkload", "WORKLOADS"]


@dataclass(frozen=True)
class ConeWorkload:
    name: str = "cone256"
    n: tuple = (256, 256, 256)
    voxel: float = 0.5
    n_view: int = 360
    det_nx: int = 512
    det_ny: int = 384
    pitch: float = 0.8
    sid: float = 1000.0
    sdd: float = 1500.0
    n_ellipsoid: int = 12
    seed: int = 0

    @property
    def n_ray(self):
        return self.n_view * self.det_nx * self.det_ny

    def geometry(self):
        from .tomography import build_conebeam_3d_geometry, standard_image_transform_3d
        src, dst = build_conebeam_3d_geometry(self.n_view, self.det_nx, self.det_ny, self.sid, self.sdd, self.pitch)
        M, b = standard_image_transform_3d(*self.n, self.voxel, self.voxel, self.voxel)
        return src, dst, M, b

    def phantom(self, device="cpu"):
        from .phantoms import ellipsoid_phantom_3d
        return ellipsoid_phantom_3d(*self.n, voxel=self.voxel, n_ellipsoid=self.n_ellipsoid, seed=self.seed,
                                    device=device)


@dataclass(frozen=True)
class FanWorkload:
    name: str = "fan256"
    n: tuple = (256, 256)
    pixel: float = 1.0
    n_view: int = 360
    n_det: int = 512
    pitch: float = 1.0
    sid: float = 1000.0
    sdd: float = 1500.0
    seed: int = 0

    @property
    def n_ray(self):
        return self.n_view * self.n_det

    def geometry(self):
        from .tomography import build_fanbeam_2d_geometry, standard_image_transform_2d
        src, dst = build_fanbeam_2d_geometry(self.n_view, self.n_det, self.sid, self.sdd, self.pitch)
        M, b = standard_image_transform_2d(*self.n, self.pixel, self.pixel)
        return src, dst, M, b

    def phantom(self, device="cpu"):
        from .phantoms import ellipse_phantom_2d
        return ellipse_phantom_2d(*self.n, pixel=self.pixel, seed=self.seed, device=device)


WORKLOADS = {"cone256": ConeWorkload(), "fan256": FanWorkload()}
