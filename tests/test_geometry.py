"""Geometry builders reproduce the reference's rays exactly (fixtures made
by the reference's own builders, tests/golden/make_golden.py).  CPU only."""
import math

import numpy as np
import torch

from conftest import load_golden
from ct_laboratory_b200.tomography import (build_circular_sequence, build_conebeam_3d_geometry,
                                           build_fanbeam_2d_geometry, build_helical_sequence,
                                           build_static_2d_geometry, build_static_3d_geometry,
                                           build_uniform_static_2d_geometry, build_uniform_static_3d_geometry,
                                           standard_image_transform_2d, standard_image_transform_3d)


def test_fanbeam_and_conebeam_rays_exact():
    g = load_golden("geometry")
    src, dst = build_fanbeam_2d_geometry(n_view=7, n_det=9, sid=500.0, sdd=800.0, det_spacing=1.3, angle_offset=0.2)
    assert np.array_equal(src.numpy(), g["fan_src"]) and np.array_equal(dst.numpy(), g["fan_dst"])
    src, dst = build_conebeam_3d_geometry(n_view=5, det_nx=6, det_ny=4, sid=500.0, sdd=800.0, det_spacing=1.3,
                                          angle_offset=0.1)
    assert np.array_equal(src.numpy(), g["cone_src"]) and np.array_equal(dst.numpy(), g["cone_dst"])
    f2 = load_golden("fan2d")
    src, dst = build_fanbeam_2d_geometry(n_view=10, n_det=48, sid=60.0, sdd=100.0, det_spacing=1.1)
    assert np.array_equal(src.numpy(), f2["src"]) and np.array_equal(dst.numpy(), f2["dst"])
    c3 = load_golden("cone3d")
    src, dst = build_conebeam_3d_geometry(n_view=6, det_nx=16, det_ny=12, sid=40.0, sdd=70.0, det_spacing=0.9)
    assert np.array_equal(src.numpy(), c3["src"]) and np.array_equal(dst.numpy(), c3["dst"])


def test_conebeam_ray_order_is_view_v_u():
    src, dst = build_conebeam_3d_geometry(n_view=3, det_nx=5, det_ny=4, sid=100.0, sdd=150.0)
    d = dst.view(3, 4, 5, 3)
    # v (rows) moves along +z, u (cols) stays in the z = 0 plane
    assert torch.all(d[:, 1:, :, 2] > d[:, :-1, :, 2])
    assert torch.allclose(d[:, :, 1:, 2], d[:, :, :-1, 2])


def test_image_transforms():
    g = load_golden("geometry")
    M2, b2 = standard_image_transform_2d(7, 5, 1.5, 2.0)
    M3, b3 = standard_image_transform_3d(7, 5, 4, 1.5, 2.0, 0.5)
    for a, k in ((M2, "M2"), (b2, "b2"), (M3, "M3"), (b3, "b3")):
        assert np.array_equal(a.numpy(), g[k])


def test_static2d_rays_exact():
    g = load_golden("static2d")
    n_frame, n_source = 3, 4
    th = torch.tensor([0.0, 0.4, 1.1])
    Mg = torch.stack([torch.tensor([[math.cos(a), -math.sin(a)], [math.sin(a), math.cos(a)]]) for a in th.tolist()])
    bg = torch.tensor([[0.0, 0.0], [0.5, -0.3], [-0.2, 0.1]])
    active = torch.zeros(n_frame, n_source, dtype=torch.bool)
    active[0, 0] = active[1, 1] = active[1, 3] = active[2, 2] = True
    sp, mc, mo, smm = build_uniform_static_2d_geometry(n_source, 40.0, 6, 34.0, 8, 2.0, Mg, bg, active)
    src, dst = build_static_2d_geometry(sp, mc, mo, 8, 2.0, smm, Mg, bg, active)
    assert np.array_equal(src.numpy(), g["src"]) and np.array_equal(dst.numpy(), g["dst"])


def test_static3d_rays_exact():
    g = load_golden("static3d_geom")
    sp, mc, mo, smm = build_uniform_static_3d_geometry(6, 40.0, 0.0, 10, 34.0, 0.5, 3, device="cpu")
    for a, k in ((sp, "source_positions"), (mc, "module_centers"), (mo, "module_orientations"),
                 (smm, "source_module_mask")):
        assert np.array_equal(a.numpy(), g[k]), k
    Mg, bg, act = build_circular_sequence(3, 6, device="cpu")
    src, dst = build_static_3d_geometry(sp, mc, mo, 4, 3, 1.2, 1.1, smm, Mg, bg, act, device="cpu")
    assert np.array_equal(src.numpy(), g["src"]) and np.array_equal(dst.numpy(), g["dst"])
    Mh, bh, acth = build_helical_sequence(4, 6, 3.0, device="cpu")
    assert np.array_equal(Mh.numpy()[:, :2, :2], np.repeat(np.eye(2, dtype=np.float32)[None], 4, 0))
    assert np.array_equal(bh.numpy(), g["bh"]) and np.array_equal(acth.numpy(), g["active_h"])
    src, dst = build_static_3d_geometry(sp, mc, mo, 4, 3, 1.2, 1.1, smm, Mh, bh, acth, device="cpu")
    assert np.array_equal(src.numpy(), g["src_h"]) and np.array_equal(dst.numpy(), g["dst_h"])


def test_empty_active_set():
    sp, mc, mo, smm = build_uniform_static_3d_geometry(2, 40.0, 0.0, 4, 34.0, 0.0, 2, device="cpu")
    Mg, bg, act = build_circular_sequence(2, 2, device="cpu")
    act[:] = False
    src, dst = build_static_3d_geometry(sp, mc, mo, 2, 2, 1.0, 1.0, smm, Mg, bg, act, device="cpu")
    assert src.shape == (0, 3) and dst.shape == (0, 3)
