"""The 2-D adjoint with transposed scratch
(ctlab_back_project_2d_siddon_ws, ScanBatch's image_scratch).

Rays whose larger index-space direction component runs along the image's
stride-1 axis accumulate into a transposed copy of the image, added back at
the end; the lanes of a warp walk row-aligned.  The segments are those of the
per-lane crossing-rule walk, so the result equals the scratch-free adjoint up
to the order of the float additions (tolerance 1e-5, the projector
tolerance), and the oracle (the reference's plane-sort walk, float32, on
the image embedded as a one-voxel-thick volume) within the same 1e-5, under
both voxel rules (the midpoint rule with the reference's segments just
outside the grid).
Images are non-square so that a mix-up of the transposed strides shows;
views cover the full circle so that every warp kind occurs (rays along rows,
along columns, near 45 degrees, mixed within a warp).
"""
import numpy as np
import pytest
import torch

from conftest import rel_err
from oracle import oracle as O

pytestmark = pytest.mark.gpu
DEV = "cuda"
TOL = 1e-5


def _fan(n_row, n_col, n_view, n_det, pixel, seed=0):
    from ct_laboratory_b200.tomography import build_fanbeam_2d_geometry, standard_image_transform_2d
    src, dst = build_fanbeam_2d_geometry(n_view, n_det, 200.0, 300.0, 0.7, angle_offset=0.1 * seed)
    M, b = standard_image_transform_2d(n_row, n_col, pixel, pixel)
    return [t.to(DEV).contiguous() for t in (src, dst, M, b)]


def _crossing_opts(n_view, n_det, rule=1):
    from ct_laboratory_b200 import _native as N
    # rays [view][cell], lanes of a warp along cells (neighbouring rays)
    return N.tiling(1, n_det, n_view, n_det * n_view, 1, n_det, tile_rows=32, block_threads=128,
                    voxel_rule=N.VOXEL_CROSSING if rule == 1 else N.VOXEL_MIDPOINT)


def _adjoint(sino, src, dst, Mi, b, n_row, n_col, opts, scratch, out=None, accumulate=0):
    from ct_laboratory_b200 import _native as N
    batch, n_ray = sino.shape
    if out is None:
        out = torch.empty((batch, n_row, n_col), device=DEV)
    N.call("ctlab_back_project_2d_siddon_ws", N.ptr(sino), batch, n_ray, N.ptr(src), N.ptr(dst), N.ptr(Mi), N.ptr(b),
           n_row, n_col, N.ptr(out), accumulate, N.tiling_ref(opts), N.ptr(scratch), N.stream_of(sino))
    torch.cuda.synchronize()
    return out


def _embed_3d(src, dst, Mi, b):
    """The 2-D geometry as a one-voxel-thick 3-D one (z = 0)."""
    z = np.zeros((src.shape[0], 1), np.float32)
    s3 = np.concatenate([src.cpu().numpy(), z], 1)
    d3 = np.concatenate([dst.cpu().numpy(), z], 1)
    M3 = np.eye(3, dtype=np.float32)
    M3[:2, :2] = Mi.cpu().numpy()
    b3 = np.concatenate([b.cpu().numpy(), [0.0]]).astype(np.float32)
    return s3, d3, M3, b3


@pytest.mark.parametrize("rule", ["crossing", "midpoint", "midpoint-flat"])
@pytest.mark.parametrize("shape", [(40, 56), (56, 40), (64, 64)])
def test_scratch_adjoint_matches_plain_and_oracle(shape, rule):
    """Both voxel rules; the midpoint rule (the reference's) also without a
    tiling (consecutive rays per warp), the projector modules' default."""
    from ct_laboratory_b200.tomography._common import inverse
    n_row, n_col = shape
    n_view, n_det = 45, 96
    src, dst, M, b = _fan(n_row, n_col, n_view, n_det, pixel=64.0 / max(shape))
    Mi = inverse(M)
    opts = None if rule == "midpoint-flat" else _crossing_opts(n_view, n_det, 1 if rule == "crossing" else 0)
    g = torch.Generator(device=DEV).manual_seed(1)
    sino = torch.rand(3, n_view * n_det, device=DEV, generator=g)
    scratch = torch.full((3, n_row, n_col), float("nan"), device=DEV)  # contents must not matter
    with_t = _adjoint(sino, src, dst, Mi, b, n_row, n_col, opts, scratch)
    plain = _adjoint(sino, src, dst, Mi, b, n_row, n_col, opts, None)
    for k in range(3):
        assert rel_err(with_t[k].cpu().numpy(), plain[k].cpu().numpy()) < TOL
    s3, d3, M3, b3 = _embed_3d(src, dst, Mi, b)
    ref = O.back_planesort(sino[1].cpu().numpy(), M3, b3, s3, d3, (n_row, n_col, 1))[..., 0]
    assert rel_err(with_t[1].cpu().numpy(), ref) < TOL


@pytest.mark.parametrize("shape", [(12, 4100), (4100, 12)])
def test_scratch_adjoint_beyond_the_major_walk_bound(shape):
    """Images wider or taller than 4096 pixels are outside the major-axis
    walk's bound: every ray takes the merge walk into the image itself, the
    scratch being zeroed and added back empty."""
    from ct_laboratory_b200.tomography._common import inverse
    n_row, n_col = shape
    n_view, n_det = 16, 64
    src, dst, M, b = _fan(n_row, n_col, n_view, n_det, pixel=0.05)
    Mi = inverse(M)
    for rule in (1, 0):
        opts = _crossing_opts(n_view, n_det, rule)
        sino = torch.rand(1, n_view * n_det, device=DEV, generator=torch.Generator(device=DEV).manual_seed(2))
        with_t = _adjoint(sino, src, dst, Mi, b, n_row, n_col, opts, torch.empty(1, n_row, n_col, device=DEV))
        plain = _adjoint(sino, src, dst, Mi, b, n_row, n_col, opts, None)
        assert rel_err(with_t[0].cpu().numpy(), plain[0].cpu().numpy()) < TOL
        if rule == 0:
            s3, d3, M3, b3 = _embed_3d(src, dst, Mi, b)
            ref = O.back_planesort(sino[0].cpu().numpy(), M3, b3, s3, d3, (n_row, n_col, 1))[..., 0]
            assert rel_err(with_t[0].cpu().numpy(), ref) < TOL


def test_scratch_adjoint_accumulates_and_is_the_transpose():
    from ct_laboratory_b200.tomography import forward_project_2d_siddon
    from ct_laboratory_b200.tomography._common import inverse
    n_row, n_col, n_view, n_det = 48, 36, 30, 80
    src, dst, M, b = _fan(n_row, n_col, n_view, n_det, pixel=1.2, seed=2)
    Mi = inverse(M)
    opts = _crossing_opts(n_view, n_det)
    g = torch.Generator(device=DEV).manual_seed(3)
    y = torch.rand(2, n_view * n_det, device=DEV, generator=g)
    x = torch.rand(2, n_row, n_col, device=DEV, generator=g)
    scratch = torch.empty(2, n_row, n_col, device=DEV)
    aty = _adjoint(y, src, dst, Mi, b, n_row, n_col, opts, scratch)
    # accumulate: out = 1 + A^T y
    out = torch.ones(2, n_row, n_col, device=DEV)
    _adjoint(y, src, dst, Mi, b, n_row, n_col, opts, scratch, out=out, accumulate=1)
    assert rel_err(out.cpu().numpy(), (1.0 + aty).cpu().numpy()) < TOL
    # <A x, y> = <x, A^T y> with the crossing-rule forward
    ax = forward_project_2d_siddon(x, Mi, b, src, dst, opts)
    lhs = float((ax.double() * y.double()).sum())
    rhs = float((x.double() * aty.double()).sum())
    assert abs(lhs - rhs) / abs(rhs) < TOL


def test_module_adjoint_uses_scratch_and_autograd_agrees():
    """The 2-D module with a crossing-rule tiling: back_project (which passes
    scratch) against the plain entry point, and the autograd gradient."""
    from ct_laboratory_b200 import CTProjector2DModule
    from ct_laboratory_b200 import _native as N
    n_row, n_col, n_view, n_det = 50, 34, 24, 64
    src, dst, M, b = _fan(n_row, n_col, n_view, n_det, pixel=1.5, seed=4)
    opts = _crossing_opts(n_view, n_det)
    p = CTProjector2DModule(n_row, n_col, M, b, src, dst, ray_tiling=opts)
    g = torch.Generator(device=DEV).manual_seed(5)
    y = torch.rand(n_view * n_det, device=DEV, generator=g)
    bp = p.back_project(y)
    plain = _adjoint(y[None], src, dst, p.M_inv, b, n_row, n_col, opts, None)[0]
    assert rel_err(bp.cpu().numpy(), plain.cpu().numpy()) < TOL
    x = torch.rand(n_row, n_col, device=DEV, generator=g, requires_grad=True)
    (p(x) * y).sum().backward()
    assert rel_err(x.grad.cpu().numpy(), plain.cpu().numpy()) < TOL
    assert N.VOXEL_CROSSING == opts.voxel_rule


def test_batched_scratch_matches_plain_per_scan_adjoint():
    """ScanBatch (transposed scratch per scan, one persistent launch, the
    add-back pass) against the scratch-free single-scan adjoint, on
    non-square images, with accumulate."""
    from ct_laboratory_b200 import CTProjector2DModule
    from ct_laboratory_b200.batched import ScanBatch
    from ct_laboratory_b200.tomography._common import inverse
    projs, geo = [], []
    for i, (n_row, n_col) in enumerate([(40, 64), (64, 40), (48, 48), (24, 72)]):
        n_view, n_det = 20 + 5 * i, 64
        src, dst, M, b = _fan(n_row, n_col, n_view, n_det, pixel=80.0 / max(n_row, n_col), seed=i)
        p = CTProjector2DModule(n_row, n_col, M, b, src, dst)
        p.n_view, p.n_det = n_view, n_det  # [view][cell] ray grid: the grid tile kinds apply
        projs.append(p)
        geo.append((src, dst, inverse(M), b, n_row, n_col, _crossing_opts(n_view, n_det)))
    for kind in ("flat", "grid32"):
        batch = ScanBatch(projs, block_threads=128, kind=kind)
        assert batch.scratch is not None
        g = torch.Generator(device=DEV).manual_seed(6)
        for s in batch.sinos_in:
            s.copy_(torch.rand(s.shape, device=DEV, generator=g))
        batch.back()
        torch.cuda.synchronize()
        first = [t.clone() for t in batch.images_out]
        for i, (src, dst, Mi, b, n_row, n_col, opts) in enumerate(geo):
            plain = _adjoint(batch.sinos_in[i][None], src, dst, Mi, b, n_row, n_col, opts, None)[0]
            assert rel_err(first[i].cpu().numpy(), plain.cpu().numpy()) < TOL, (kind, i)
        batch.back(accumulate=True)
        torch.cuda.synchronize()
        for i in range(len(projs)):
            assert rel_err(batch.images_out[i].cpu().numpy(), (2 * first[i]).cpu().numpy()) < TOL, (kind, i)


def test_scratch_must_not_alias_output():
    from ct_laboratory_b200 import _native as N
    from ct_laboratory_b200.tomography._common import inverse
    src, dst, M, b = _fan(16, 16, 4, 32, pixel=4.0)
    out = torch.empty(1, 16, 16, device=DEV)
    sino = torch.rand(1, 4 * 32, device=DEV)
    with pytest.raises(RuntimeError, match="scratch"):
        N.call("ctlab_back_project_2d_siddon_ws", N.ptr(sino), 1, 4 * 32, N.ptr(src), N.ptr(dst), N.ptr(inverse(M)),
               N.ptr(b), 16, 16, N.ptr(out), 0, N.tiling_ref(_crossing_opts(4, 32)), N.ptr(out), N.stream_of(sino))
