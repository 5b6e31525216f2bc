"""The column walk with two 16-lane groups per warp (detectors with 16 rows
per column, StaticCT modules tiled by staticct_ray_tiling) against the
per-lane walk, under the crossing rule.

The column walk takes the per-lane walk's segments in the same order, so the
forward is bitwise equal to it; the adjoint agrees up to the order of the
float atomic additions (projector tolerance 1e-5).  The small ring below is
built so that every case the two-group walk handles occurs: rays leaving
through the volume's top or bottom (non-uniform groups), rays missing the
volume, groups whose 16 rays all miss next to a group that walks, and
groups of different lengths in one warp.
"""
import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu
DEV = "cuda"
TOL = 1e-5


def _ring():
    from ct_laboratory_b200.tomography import UniformStaticCTProjector3D, standard_image_transform_3d
    n = (40, 36, 20)
    M, b = standard_image_transform_3d(*n, 1.0, 1.0, 0.25)  # a thin slab: the outer rows miss it
    n_frame, n_source = 2, 6
    Mg = torch.stack([torch.eye(3), torch.tensor([[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])])
    bg = torch.zeros(n_frame, 3)
    act = torch.ones(n_frame, n_source, dtype=torch.bool)
    p = UniformStaticCTProjector3D(*n, n_source, 60.0, 0.0, 12, 55.0, 8, 16, 3.0, 1.5, 0.0, Mg, bg, act, 4, M, b,
                                   device=torch.device(DEV))
    return p, n, n_frame * n_source * 4


@pytest.mark.parametrize("batch", [1, 3, 5])  # 1, 2 and 4 volumes per walk (and a partial last group)
def test_two_group_column_walk_equals_per_lane_walk(batch):
    from ct_laboratory_b200 import _C
    from ct_laboratory_b200 import _native as N
    from ct_laboratory_b200.tomography import staticct_ray_tiling
    p, n, n_view = _ring()
    src, dst, b = p.src, p.dst, p.b
    Mi = torch.inverse(p.M).contiguous()
    tiled = staticct_ray_tiling(n_view, 8, 16, voxel_rule=N.VOXEL_CROSSING)
    assert tiled is not None and tiled.tile_rows == 16
    flat = N.flat_opts(voxel_rule=N.VOXEL_CROSSING, block_threads=128)
    g = torch.Generator(device=DEV).manual_seed(3)
    x = torch.rand(batch, *n, device=DEV, generator=g)
    y = torch.rand(batch, src.shape[0], device=DEV, generator=g)

    f16 = _C.forward_project_3d_on_the_fly_cuda(x, src, dst, Mi, b, tiling=tiled)
    f1 = _C.forward_project_3d_on_the_fly_cuda(x, src, dst, Mi, b, tiling=flat)
    assert torch.equal(f16, f1)

    # the geometry covers the cases the two-group walk must handle
    hit = (f1[0] != 0).reshape(-1, 16)  # one row per 16-ray group (a module column)
    per_group = hit.sum(1)
    pairs = per_group.reshape(-1, 2)  # the two groups of a warp
    assert bool(((pairs[:, 0] == 0) & (pairs[:, 1] > 0)).any() | ((pairs[:, 1] == 0) & (pairs[:, 0] > 0)).any())
    assert bool(((per_group > 0) & (per_group < 16)).any())  # partly missing groups

    b16 = _C.back_project_3d_on_the_fly_cuda(y, src, dst, Mi, b, *n, tiling=tiled)
    b1 = _C.back_project_3d_on_the_fly_cuda(y, src, dst, Mi, b, *n, tiling=flat)
    for k in range(batch):
        assert rel_err(b16[k].cpu().numpy(), b1[k].cpu().numpy()) < TOL


def test_static_module_takes_the_tiling():
    """UniformStaticCTProjector3D with the tiling: forward bitwise the flat
    module's, and autograd through it."""
    from ct_laboratory_b200 import CTProjector3DModule
    from ct_laboratory_b200 import _native as N
    from ct_laboratory_b200.tomography import UniformStaticCTProjector3D, staticct_ray_tiling
    p, n, n_view = _ring()
    tiled = UniformStaticCTProjector3D(*n, 6, 60.0, 0.0, 12, 55.0, 8, 16, 3.0, 1.5, 0.0, p.M_gantry, p.b_gantry,
                                       p.active_sources, 4, p.M, p.b, device=torch.device(DEV),
                                       ray_tiling=staticct_ray_tiling(n_view, 8, 16, voxel_rule=N.VOXEL_CROSSING))
    flat = CTProjector3DModule(*n, p.M, p.b, p.src, p.dst, device=torch.device(DEV),
                               ray_tiling=N.flat_opts(voxel_rule=N.VOXEL_CROSSING))
    x = torch.rand(*n, device=DEV, requires_grad=True)
    assert torch.equal(tiled(x), flat(x))
    auto = UniformStaticCTProjector3D(*n, 6, 60.0, 0.0, 12, 55.0, 8, 16, 3.0, 1.5, 0.0, p.M_gantry, p.b_gantry,
                                      p.active_sources, 4, p.M, p.b, device=torch.device(DEV), voxel_rule=1)
    assert auto.ray_tiling.tile_rows == 16 and torch.equal(auto(x), flat(x))
    yv = torch.rand(p.src.shape[0], device=DEV)
    (tiled(x) * yv).sum().backward()
    assert rel_err(x.grad.cpu().numpy(), flat.back_project(yv).cpu().numpy()) < TOL
