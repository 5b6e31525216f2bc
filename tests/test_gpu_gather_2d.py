"""The deterministic 2-D adjoint (back_project_2d_gather_cuda, the 2-D
modules' ``deterministic_adjoint=True``).

It gathers per pixel through the 3-D gather kernel, the image being the
one-voxel-thick volume [n_row, n_col, 1] with the rays in its z = 0 plane,
where the 3-D arithmetic reduces exactly to the 2-D walk's.  So it must be:
bitwise reproducible from call to call; the crossing-rule atomic adjoint
up to the rounding of the products (y * |v| * span grouped differently) and
the order of the float additions (tolerance 1e-6 here, well inside the
projector tolerance 1e-5); the transpose of the crossing-rule forward
(<A x, y> = <x, A^T y> in FP64 accumulation to 1e-6); and what autograd
returns as the gradient, bitwise.
"""
import math

import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _crossing_adjoint(p, y, n_view, n_det):
    from ct_laboratory_b200 import _native as N
    from ct_laboratory_b200.tomography import back_project_2d_siddon
    opts = N.tiling(1, n_det, n_view, n_det * n_view, 1, n_det, tile_rows=32, block_threads=128,
                    voxel_rule=N.VOXEL_CROSSING)
    return back_project_2d_siddon(y, p.M_inv, p.b, p.src, p.dst, p.n_row, p.n_col, opts), opts


def test_fan_gather_adjoint():
    from ct_laboratory_b200 import FanBeam2DProjector
    from ct_laboratory_b200.tomography import forward_project_2d_siddon
    n_row, n_col, n_view, n_det = 52, 40, 36, 80
    p = FanBeam2DProjector(n_row, n_col, n_view=n_view, n_det=n_det, sid=120.0, sdd=180.0, det_spacing=0.9,
                           pixel_size=1.1, device=torch.device(DEV), deterministic_adjoint=True)
    g = torch.Generator(device=DEV).manual_seed(1)
    y = torch.rand(3, n_view * n_det, device=DEV, generator=g)
    a1 = p.back_project(y)
    a2 = p.back_project(y)
    assert a1.shape == (3, n_row, n_col) and torch.equal(a1, a2)
    atomic, opts = _crossing_adjoint(p, y, n_view, n_det)
    for k in range(3):
        assert rel_err(a1[k].cpu().numpy(), atomic[k].cpu().numpy()) < 1e-6
    x = torch.rand(n_row, n_col, device=DEV, generator=g)
    ax = forward_project_2d_siddon(x, p.M_inv, p.b, p.src, p.dst, opts)[0]
    lhs = float((ax.double() * y[0].double()).sum())
    rhs = float((x.double() * a1[0].double()).sum())
    assert abs(lhs - rhs) / abs(rhs) < 1e-6
    # autograd: the backward is the gather
    xg = x.clone().requires_grad_(True)
    (p(xg) * y[1]).sum().backward()
    assert torch.equal(xg.grad, a1[1])


def test_static_ring_gather_adjoint():
    from ct_laboratory_b200 import UniformStaticCTProjector2D
    from ct_laboratory_b200 import _native as N
    from ct_laboratory_b200.tomography import back_project_2d_siddon, standard_image_transform_2d
    n = 48
    M, b = standard_image_transform_2d(n, n, 1.0, 1.0)
    n_frame, n_source = 2, 6
    Mg = torch.stack([torch.tensor([[math.cos(0.1 * f), -math.sin(0.1 * f)],
                                    [math.sin(0.1 * f), math.cos(0.1 * f)]]) for f in range(n_frame)])
    act = torch.ones(n_frame, n_source, dtype=torch.bool)
    p = UniformStaticCTProjector2D(n, n, M, b, n_source, 90.0, 8, 85.0, 16, 1.0, Mg, torch.zeros(n_frame, 2), act,
                                   device=torch.device(DEV), deterministic_adjoint=True)
    y = torch.rand(p.src.shape[0], device=DEV, generator=torch.Generator(device=DEV).manual_seed(4))
    a1 = p.back_project(y)
    assert torch.equal(a1, p.back_project(y))
    atomic = back_project_2d_siddon(y, p.M_inv, p.b, p.src, p.dst, n, n,
                                    N.flat_opts(voxel_rule=N.VOXEL_CROSSING))[0]
    assert rel_err(a1.cpu().numpy(), atomic.cpu().numpy()) < 1e-6


def test_gather_needs_panels():
    from ct_laboratory_b200 import CTProjector2DModule
    with pytest.raises(ValueError, match="panels"):
        CTProjector2DModule(8, 8, torch.eye(2, device=DEV), torch.zeros(2, device=DEV), torch.zeros(4, 2, device=DEV),
                            torch.ones(4, 2, device=DEV), deterministic_adjoint=True)
