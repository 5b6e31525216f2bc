"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run in a container that has the reference checkout (read-only) at
``$CTLAB_REFERENCE`` (else the checkout beside this repository)::

    python tests/golden/make_golden.py

It imports the reference's pure-PyTorch projector path and its geometry
builders directly from the checkout (the compiled ``ct_laboratory._C`` is
replaced by an empty stub: nothing here calls CUDA) and stores, for small
seeded cases, the reference's own outputs as ``.npz`` files.  The fixtures
are committed; the GPU box never needs the reference checkout.

Cases
-----
kat2d / kat3d   the reference's two single-ray known answers
                (python_examples/test_ct_projector_2d_line_integral.py:31-43,70,
                 test_ct_projector_3d_line_integral.py:33-45,74)
fan2d           FanBeam geometry, non-square image, non-power-of-2 pixels
cone3d          ConeBeam geometry, non-cubic volume, 0.7 mm voxels, plus the
                uint16 compressor and the compressed-tvals projector
affine3d        non-diagonal voxel->world affine, random rays
edge3d          axis-parallel rays, rays starting inside, rays that miss
static2d        UniformStaticCTProjector2D ring with rotating frames
static3d        uniform StaticCT 3-D ring (farthest-module mask), circular and
                helical frame sequences
"""
from __future__ import annotations

import importlib
import math
import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.reference_path import reference_root  # noqa: E402

REF = reference_root(required=True)


def load_reference():
    """Import ct_laboratory.tomography modules from the checkout without
    running the package __init__ (which needs the compiled extension)."""
    pkg_dir = os.path.join(REF, "ct_laboratory")
    root = types.ModuleType("ct_laboratory")
    root.__path__ = [pkg_dir]
    sys.modules["ct_laboratory"] = root
    sys.modules["ct_laboratory._C"] = types.ModuleType("ct_laboratory._C")
    tomo = types.ModuleType("ct_laboratory.tomography")
    tomo.__path__ = [os.path.join(pkg_dir, "tomography")]
    sys.modules["ct_laboratory.tomography"] = tomo
    mods = {}
    for name in ("ct_projector_2d_torch", "ct_projector_3d_torch", "standard_image_transform",
                 "fanbeam_projector_2d", "conebeam_projector_3d", "staticct_projector_2d",
                 "staticct_projector_3d"):
        mods[name] = importlib.import_module("ct_laboratory.tomography." + name)
    return mods


def np32(t):
    return t.detach().cpu().numpy().astype(np.float32) if t.dtype.is_floating_point else t.detach().cpu().numpy()


def ellipse_image(n_row, n_col, seed):
    g = torch.Generator().manual_seed(seed)
    r = torch.arange(n_row, dtype=torch.float32)[:, None] / n_row - 0.5
    c = torch.arange(n_col, dtype=torch.float32)[None, :] / n_col - 0.5
    img = torch.zeros(n_row, n_col)
    for _ in range(5):
        cr, cc = (torch.rand(2, generator=g) - 0.5) * 0.5
        ar, ac = torch.rand(2, generator=g) * 0.3 + 0.05
        img += torch.rand(1, generator=g) * 0.02 * (((r - cr) / ar) ** 2 + ((c - cc) / ac) ** 2 <= 1).float()
    return img.contiguous()


def ellipsoid_volume(shape, seed):
    g = torch.Generator().manual_seed(seed)
    axes = [torch.arange(n, dtype=torch.float32) / n - 0.5 for n in shape]
    X, Y, Z = torch.meshgrid(*axes, indexing="ij")
    vol = torch.zeros(shape)
    for _ in range(4):
        c = (torch.rand(3, generator=g) - 0.5) * 0.5
        a = torch.rand(3, generator=g) * 0.3 + 0.08
        inside = ((X - c[0]) / a[0]) ** 2 + ((Y - c[1]) / a[1]) ** 2 + ((Z - c[2]) / a[2]) ** 2 <= 1
        vol += torch.rand(1, generator=g) * 0.02 * inside.float()
    return vol.contiguous()


def run_2d(m, name, n_row, n_col, M, b, src, dst, img, y):
    t2 = m["ct_projector_2d_torch"]
    tv = t2.compute_intersections_2d_torch(n_row, n_col, M, b, src, dst)
    fwd = t2.forward_project_2d_torch(img, tv, M, b, src, dst)
    back = t2.back_project_2d_torch(y, tv, M, b, src, dst, n_row, n_col)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), dims=np.array([n_row, n_col], np.int32),
                        M=np32(M), Minv=np32(torch.inverse(M)), b=np32(b), src=np32(src), dst=np32(dst),
                        img=np32(img), y=np32(y), tvals=np32(tv), fwd=np32(fwd), back=np32(back))
    return fwd


def run_3d(m, name, dims, M, b, src, dst, vol, y, compressed=False):
    t3 = m["ct_projector_3d_torch"]
    nx, ny, nz = dims
    tv = t3.compute_intersections_3d_torch(nx, ny, nz, M, b, src, dst)
    fwd = t3.forward_project_3d_torch(vol, tv, M, b, src, dst)
    back = t3.back_project_3d_torch(y, tv, M, b, src, dst, nx, ny, nz)
    out = dict(dims=np.array(dims, np.int32), M=np32(M), Minv=np32(torch.inverse(M)), b=np32(b), src=np32(src),
               dst=np32(dst), vol=np32(vol), y=np32(y), tvals=np32(tv), fwd=np32(fwd), back=np32(back))
    if compressed:
        u16, starts, scales = t3.compress_tvals_to_uint16(tv, M, src, dst)
        diags = torch.tensor([[1, 1, 1], [1, 1, -1], [1, -1, 1], [-1, 1, 1]], dtype=M.dtype).t()
        vdl = torch.norm(M @ diags, dim=0).max()
        out.update(u16=u16.numpy().view(np.uint16), starts=np32(starts), scales=np32(scales),
                   voxel_diag=np.float32(vdl.item()),
                   decomp=np32(t3.decompress_tvals_from_uint16(u16, starts, scales)),
                   fwd_comp=np32(t3.forward_project_3d_torch(vol, (u16, starts, scales), M, b, src, dst)),
                   back_comp=np32(t3.back_project_3d_torch(y, (u16, starts, scales), M, b, src, dst, nx, ny, nz)))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    return fwd


def main():
    torch.set_num_threads(1)
    m = load_reference()
    sit = m["standard_image_transform"]

    # --- known answers ---------------------------------------------------
    img = torch.zeros(32, 32)
    img[16, :] = 1.0
    run_2d(m, "kat2d", 32, 32, torch.eye(2), torch.zeros(2), torch.tensor([[16.0, -5.0]]),
           torch.tensor([[16.0, 37.0]]), img, torch.ones(1))
    vol = torch.zeros(32, 32, 32)
    vol[:, 16, 16] = 1.0
    run_3d(m, "kat3d", (32, 32, 32), torch.eye(3), torch.zeros(3), torch.tensor([[200.0, 16.0, 16.0]]),
           torch.tensor([[-200.0, 16.0, 16.0]]), vol, torch.ones(1))

    # --- fan-beam 2-D ----------------------------------------------------
    fb = m["fanbeam_projector_2d"]
    src, dst = fb.build_fanbeam_2d_geometry(n_view=10, n_det=48, sid=60.0, sdd=100.0, det_spacing=1.1)
    M, b = sit.standard_image_transform_2d(40, 36, 0.9, 0.9)
    g = torch.Generator().manual_seed(7)
    run_2d(m, "fan2d", 40, 36, M, b, src, dst, ellipse_image(40, 36, 1),
           torch.rand(src.shape[0], generator=g))

    # --- cone-beam 3-D with compression -----------------------------------
    cb = m["conebeam_projector_3d"]
    src, dst = cb.build_conebeam_3d_geometry(n_view=6, det_nx=16, det_ny=12, sid=40.0, sdd=70.0, det_spacing=0.9)
    M, b = sit.standard_image_transform_3d(14, 12, 10, 0.7, 0.7, 0.7)
    g = torch.Generator().manual_seed(11)
    run_3d(m, "cone3d", (14, 12, 10), M, b, src, dst, ellipsoid_volume((14, 12, 10), 2),
           torch.rand(src.shape[0], generator=g), compressed=True)

    # --- general affine, random rays --------------------------------------
    g = torch.Generator().manual_seed(13)
    ang = 0.3
    R = torch.tensor([[math.cos(ang), -math.sin(ang), 0.0], [math.sin(ang), math.cos(ang), 0.0], [0.0, 0.0, 1.0]])
    M = (R @ torch.diag(torch.tensor([0.8, 1.1, 0.6]))).float()
    b = torch.tensor([-3.0, -4.5, -2.0])
    n = 300
    dirs = torch.randn(n, 3, generator=g)
    dirs = dirs / dirs.norm(dim=1, keepdim=True)
    centre = (torch.rand(n, 3, generator=g) - 0.5) * 12.0
    src, dst = centre - 30.0 * dirs, centre + 30.0 * dirs
    run_3d(m, "affine3d", (10, 9, 8), M, b, src.contiguous(), dst.contiguous(), ellipsoid_volume((10, 9, 8), 3),
           torch.rand(n, generator=g), compressed=True)

    # --- edge cases --------------------------------------------------------
    dims = (8, 7, 6)
    M, b = sit.standard_image_transform_3d(*dims, 1.0, 1.0, 1.0)
    lo = -(torch.tensor(dims, dtype=torch.float32) - 1) / 2
    rays = [
        ([-20.0, 0.0, 0.0], [20.0, 0.0, 0.0]),          # along x through the centre
        ([0.0, -20.0, 0.25], [0.0, 20.0, 0.25]),        # along y
        ([0.3, 0.2, -20.0], [0.3, 0.2, 20.0]),          # along z
        ([0.0, 0.0, 0.0], [15.0, 7.0, 3.0]),            # starts inside the volume
        ([0.5, 0.5, 0.5], [-0.5, -0.5, -0.5]),          # wholly inside
        ([-20.0, 30.0, 0.0], [20.0, 30.0, 0.0]),        # misses
        ([1.0, 1.0, 1.0], [1.0, 1.0, 1.0]),             # zero length
        ([-20.0, -20.0, -20.0], [20.0, 20.0, 20.0]),    # body diagonal (corner crossings)
        ([float(lo[0]) - 5, 0.5, 0.0], [float(-lo[0]) + 5, 0.5, 0.0]),  # along x on a y plane
        ([20.0, 0.1, 0.2], [-20.0, 0.1, 0.2]),          # negative x direction
    ]
    src = torch.tensor([r[0] for r in rays])
    dst = torch.tensor([r[1] for r in rays])
    run_3d(m, "edge3d", dims, M, b, src, dst, ellipsoid_volume(dims, 4), torch.rand(len(rays), generator=g))

    # --- StaticCT 2-D ring --------------------------------------------------
    s2 = m["staticct_projector_2d"]
    n_frame, n_source = 3, 4
    th = torch.tensor([0.0, 0.4, 1.1])
    Mg = torch.stack([torch.tensor([[math.cos(a), -math.sin(a)], [math.sin(a), math.cos(a)]]) for a in th.tolist()])
    bg = torch.tensor([[0.0, 0.0], [0.5, -0.3], [-0.2, 0.1]])
    active = torch.zeros(n_frame, n_source, dtype=torch.bool)
    active[0, 0] = active[1, 1] = active[1, 3] = active[2, 2] = True
    sp, mc, mo, smm = s2.build_uniform_static_2d_geometry(n_source, 40.0, 6, 34.0, 8, 2.0, Mg, bg, active)
    src, dst = s2.build_static_2d_geometry(sp, mc, mo, 8, 2.0, smm, Mg, bg, active)
    M, b = sit.standard_image_transform_2d(24, 24, 1.5, 1.5)
    run_2d(m, "static2d", 24, 24, M, b, src, dst, ellipse_image(24, 24, 5), torch.rand(src.shape[0], generator=g))

    # --- StaticCT 3-D ring ---------------------------------------------------
    s3 = m["staticct_projector_3d"]
    sp, mc, mo, smm = s3.build_uniform_static_3d_geometry(6, 40.0, 0.0, 10, 34.0, 0.5, 3, device="cpu")
    Mg, bg, act = s3.build_circular_sequence(3, 6, device="cpu")
    src, dst = s3.build_static_3d_geometry(sp, mc, mo, 4, 3, 1.2, 1.1, smm, Mg, bg, act, device="cpu")
    Mh, bh, acth = s3.build_helical_sequence(4, 6, 3.0, device="cpu")
    src_h, dst_h = s3.build_static_3d_geometry(sp, mc, mo, 4, 3, 1.2, 1.1, smm, Mh, bh, acth, device="cpu")
    M, b = sit.standard_image_transform_3d(12, 12, 6, 1.8, 1.8, 1.5)
    run_3d(m, "static3d", (12, 12, 6), M, b, src, dst, ellipsoid_volume((12, 12, 6), 6),
           torch.rand(src.shape[0], generator=g))
    np.savez_compressed(os.path.join(HERE, "static3d_geom.npz"), source_positions=np32(sp), module_centers=np32(mc),
                        module_orientations=np32(mo), source_module_mask=smm.numpy(), src=np32(src),
                        dst=np32(dst), Mh=np32(Mh), bh=np32(bh), active_h=acth.numpy(), src_h=np32(src_h),
                        dst_h=np32(dst_h))

    # --- geometry-builder fixtures (src/dst only) --------------------------
    src, dst = fb.build_fanbeam_2d_geometry(n_view=7, n_det=9, sid=500.0, sdd=800.0, det_spacing=1.3,
                                            angle_offset=0.2)
    s3c, d3c = cb.build_conebeam_3d_geometry(n_view=5, det_nx=6, det_ny=4, sid=500.0, sdd=800.0, det_spacing=1.3,
                                             angle_offset=0.1)
    M2, b2 = sit.standard_image_transform_2d(7, 5, 1.5, 2.0)
    M3, b3 = sit.standard_image_transform_3d(7, 5, 4, 1.5, 2.0, 0.5)
    np.savez_compressed(os.path.join(HERE, "geometry.npz"), fan_src=np32(src), fan_dst=np32(dst), cone_src=np32(s3c),
                        cone_dst=np32(d3c), M2=np32(M2), b2=np32(b2), M3=np32(M3), b3=np32(b3))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
