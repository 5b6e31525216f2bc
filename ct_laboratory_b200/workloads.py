"""Named benchmark workloads (synthetic data with the configurations' shapes).

cone256  3-D cone-beam: 256^3 volume, 0.5 mm voxels; 360 views over 360
         degrees on a circular orbit; 512 x 384 detector at 0.8 mm;
         SID 1000 mm, SDD 1500 mm; 12 seeded ellipsoids, 0-0.02/mm.
         70,778,880 rays ordered [view][det_v][det_u].
fan256   2-D fan-beam: 256^2 image, 1 mm pixels; 360 views; 512 bins at
         1 mm; SID 1000 mm, SDD 1500 mm; water disk + 10 seeded ellipses.
         184,320 rays ordered [view][bin].
batch64  64 seeded 2-D scans of uneven size: image side uniform over
         {128, 192, 256, 384, 512} (pixel = 256 mm / side, so every image
         covers the same 256 mm field), views uniform over 90-720, half
         fan-beam as fan256 (512 bins at 1 mm, SID 1000, SDD 1500), half
         StaticCT rings: 16-64 sources on a 380 mm ring, 64 modules x 16
         cells = 1024-cell arc detector on a 366.7 mm ring, views =
         frames x sources with the gantry stepped between frames.
serve    MAP reconstruction jobs arriving as a seeded Poisson process (mean
         20 jobs/s): cone-beam volumes of 128^3 / 256^3 / 384^3 (probabilities
         0.5 / 0.35 / 0.15) at 0.5 mm, 180-720 views of a 2n x 1.5n detector
         at 0.8 mm (the cone256 proportions), 20-50 iterations, I0 log-uniform
         over 1e4-1e6, quadratic smoothness prior weight 1e-2.
"""
from __future__ import annotations

import importlib
import importlib.util
import os
import sys
from dataclasses import dataclass

__all__ = ["ConeWorkload", "FanWorkload", "ScanBatchWorkload", "ServingWorkload", "StaticRingWorkload", "WORKLOADS"]

_HERE = os.path.dirname(os.path.abspath(__file__))


def _sibling(rel):
    """A self-contained module of this package (ray_geometry, phantoms,
    tomography/standard_image_transform): imported through the package when
    this file was, else loaded by file path, so that a process that loads
    this file by path (the reference CPU arm of bench.py) builds the
    workloads' rays and phantoms without mapping the native library."""
    if __package__:
        return importlib.import_module(f"{__package__}." + rel.replace("/", "."))
    name = "_ctlab_" + rel.replace("/", "_")
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(name, os.path.join(_HERE, rel + ".py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


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
        src, dst = _sibling("ray_geometry").build_conebeam_3d_geometry(self.n_view, self.det_nx, self.det_ny,
                                                                       self.sid, self.sdd, self.pitch)
        M, b = _sibling("tomography/standard_image_transform").standard_image_transform_3d(
            *self.n, self.voxel, self.voxel, self.voxel)
        return src, dst, M, b

    def phantom(self, device="cpu"):
        return _sibling("phantoms").ellipsoid_phantom_3d(*self.n, voxel=self.voxel, n_ellipsoid=self.n_ellipsoid,
                                                         seed=self.seed, device=device)


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
        src, dst = _sibling("ray_geometry").build_fanbeam_2d_geometry(self.n_view, self.n_det, self.sid, self.sdd,
                                                                      self.pitch)
        M, b = _sibling("tomography/standard_image_transform").standard_image_transform_2d(*self.n, self.pixel,
                                                                                          self.pixel)
        return src, dst, M, b

    def phantom(self, device="cpu"):
        return _sibling("phantoms").ellipse_phantom_2d(*self.n, pixel=self.pixel, seed=self.seed, device=device)


@dataclass(frozen=True)
class ScanBatchWorkload:
    name: str = "batch64"
    n_scan: int = 64
    sides: tuple = (128, 192, 256, 384, 512)
    views: tuple = (90, 720)
    sources: tuple = (16, 64)
    fov: float = 256.0
    seed: int = 0

    def instances(self):
        """One dict per scan: kind ('fan' / 'ring'), side, pixel, views and,
        for rings, sources and frames."""
        import numpy as np
        rng = np.random.default_rng(self.seed)
        out = []
        for i in range(self.n_scan):
            side = int(rng.choice(self.sides))
            views = int(rng.integers(self.views[0], self.views[1] + 1))
            d = {"kind": "fan" if i % 2 == 0 else "ring", "side": side, "pixel": self.fov / side, "views": views}
            if d["kind"] == "ring":
                n_source = int(rng.integers(self.sources[0], self.sources[1] + 1))
                d["sources"] = n_source
                d["frames"] = max(1, round(views / n_source))
                d["views"] = d["sources"] * d["frames"]
            out.append(d)
        return out

    def projectors(self, device):
        """The scans' projector modules, built on the host (the ring builder
        runs many small tensor operations) and moved to `device`."""
        import math

        import torch

        from .tomography import FanBeam2DProjector, UniformStaticCTProjector2D, standard_image_transform_2d
        out = []
        for d in self.instances():
            side, pixel = d["side"], d["pixel"]
            if d["kind"] == "fan":
                p = FanBeam2DProjector(side, side, n_view=d["views"], n_det=512, sid=1000.0, sdd=1500.0,
                                       det_spacing=1.0, pixel_size=pixel, device=torch.device("cpu"))
                out.append(p.to(device))
                continue
            n_source, n_frame = d["sources"], d["frames"]
            step = 2 * math.pi / (n_source * n_frame)
            Mg = torch.stack([torch.tensor([[math.cos(f * step), -math.sin(f * step)],
                                            [math.sin(f * step), math.cos(f * step)]], dtype=torch.float32)
                              for f in range(n_frame)])
            bg = torch.zeros(n_frame, 2)
            act = torch.ones(n_frame, n_source, dtype=torch.bool)
            M, b = standard_image_transform_2d(side, side, pixel, pixel)
            p = UniformStaticCTProjector2D(side, side, M, b, n_source, 380.0, 64, 366.7, 16,
                                           2 * math.pi * 366.7 / 1024, Mg, bg, act, device=torch.device("cpu"))
            out.append(p.to(device))
        return out

    def phantoms(self, device="cpu"):
        from .phantoms import ellipse_phantom_2d
        return [ellipse_phantom_2d(d["side"], d["side"], pixel=d["pixel"], seed=self.seed + 1 + i, device=device)
                for i, d in enumerate(self.instances())]


@dataclass(frozen=True)
class ServingWorkload:
    """MAP reconstruction requests arriving as a seeded Poisson process."""
    name: str = "serve"
    n_jobs: int = 100
    rate: float = 20.0
    sizes: tuple = (128, 256, 384)
    probs: tuple = (0.5, 0.35, 0.15)
    views: tuple = (180, 720)
    iters: tuple = (20, 50)
    I0: tuple = (1e4, 1e6)
    prior_w: float = 1e-2
    voxel: float = 0.5
    pitch: float = 0.8
    seed: int = 0

    def jobs(self):
        """One dict per job (JobSpec fields; lr is set when the request is made)."""
        import numpy as np
        rng = np.random.default_rng(self.seed)
        t = np.cumsum(rng.exponential(1.0 / self.rate, size=self.n_jobs))
        t -= t[0]
        out = []
        for i in range(self.n_jobs):
            n = int(rng.choice(self.sizes, p=self.probs))
            out.append({"job_id": i, "arrival_s": float(t[i]), "n": n,
                        "views": int(rng.integers(self.views[0], self.views[1] + 1)),
                        "iters": int(rng.integers(self.iters[0], self.iters[1] + 1)),
                        "I0": float(10 ** rng.uniform(np.log10(self.I0[0]), np.log10(self.I0[1]))),
                        "lr": 0.0, "det_nx": 2 * n, "det_ny": 3 * n // 2, "voxel": self.voxel,
                        "pitch": self.pitch, "prior_w": self.prior_w})
        return out


@dataclass(frozen=True)
class StaticRingWorkload:
    """A StaticCT ring the size of the reference's published benchmark scan
    (80 sources x 3 gantry rotations = 240 views, 16 active modules of 48 x 16
    cells per source = 12,288 cells per view, 2,949,120 rays; 512^2 x 64 voxels
    over a 400 mm x 60 mm field shifted 5 mm in z).  The calibrated geometry
    file behind the published numbers is not available, so the ring is the
    uniform one: 48 modules on a 400 mm radius, sources on a 420 mm radius,
    1.0 x 4.0 mm cells, rotations of 0, 1.5 and 3 degrees."""
    name: str = "static512"
    n: tuple = (512, 512, 64)
    fov_xy: float = 400.0
    fov_z: float = 60.0
    z_shift: float = 5.0
    n_source: int = 80
    source_radius: float = 420.0
    n_module: int = 48
    module_radius: float = 400.0
    det_nx: int = 48
    det_ny: int = 16
    pitch_x: float = 1.0
    pitch_y: float = 4.0
    modules_per_source: int = 16
    rotations_deg: tuple = (0.0, 1.5, 3.0)
    n_ellipsoid: int = 12
    seed: int = 0

    @property
    def n_ray(self):
        return self.n_source * len(self.rotations_deg) * self.modules_per_source * self.det_nx * self.det_ny

    @property
    def voxel(self):
        return (self.fov_xy / self.n[0], self.fov_xy / self.n[1], self.fov_z / self.n[2])

    @property
    def n_view(self):
        """(rotation, source) pairs, each a contiguous run of rays."""
        return self.n_source * len(self.rotations_deg)

    def geometry(self):
        """src, dst, M, b on the host."""
        import torch
        p = self.projector(torch.device("cpu"))
        return p.src, p.dst, p.M, p.b

    def projector(self, device, voxel_rule=0, deterministic_adjoint=False):
        import math

        import torch

        from .tomography import UniformStaticCTProjector3D, standard_image_transform_3d
        M, b = standard_image_transform_3d(*self.n, *self.voxel)
        b = b + torch.tensor([0.0, 0.0, self.z_shift])
        rots = []
        for deg in self.rotations_deg:
            c, s = math.cos(math.radians(deg)), math.sin(math.radians(deg))
            rots.append(torch.tensor([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]], dtype=torch.float32))
        Mg = torch.stack(rots)
        bg = torch.zeros(len(rots), 3)
        act = torch.ones(len(rots), self.n_source, dtype=torch.bool)
        return UniformStaticCTProjector3D(*self.n, self.n_source, self.source_radius, 0.0, self.n_module,
                                          self.module_radius, self.det_nx, self.det_ny, self.pitch_x, self.pitch_y,
                                          0.0, Mg, bg, act, self.modules_per_source, M, b, device=device,
                                          voxel_rule=voxel_rule, deterministic_adjoint=deterministic_adjoint)

    def phantom(self, device="cpu"):
        from .phantoms import ellipsoid_phantom_3d
        return ellipsoid_phantom_3d(*self.n, voxel=self.voxel[0], n_ellipsoid=self.n_ellipsoid, seed=self.seed,
                                    device=device)


WORKLOADS = {"cone256": ConeWorkload(), "fan256": FanWorkload(), "batch64": ScanBatchWorkload(),
             "serve": ServingWorkload(), "static512": StaticRingWorkload()}
