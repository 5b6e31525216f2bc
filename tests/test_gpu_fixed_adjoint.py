"""The reproducible 3-D adjoint (64-bit fixed-point scatter,
ctlab_back_project_3d_fixed).

Bar: bitwise the same on every call and for a sinogram alone or inside a
batch; within 1e-6 (max-normalised) of the float-atomic adjoint of the same
walk, whose own run-to-run spread is of that order; within the projector
tolerance 1e-5 of the oracle under the reference's midpoint rule; the
transpose of the forward (adjoint identity in float64, 1e-6).  Every walk
that the float adjoint takes is covered: the column walk under both voxel
rules with 32- and 16-row columns, and the per-lane walk for flat ray lists.
"""
import numpy as np
import pytest
import torch

from conftest import rel_err
from oracle import oracle as O

pytestmark = pytest.mark.gpu
DEV = "cuda"
TOL = 1e-5
TOL_FLOAT = 1e-6


def T(a):
    return torch.as_tensor(np.ascontiguousarray(a)).to(DEV, torch.float32)


def case(n=(40, 36, 28), n_view=12, det=(48, 40), pitch=0.6, seed=0):
    from ct_laboratory_b200.tomography import build_conebeam_3d_geometry, standard_image_transform_3d
    src, dst = build_conebeam_3d_geometry(n_view, det[0], det[1], 120.0, 180.0, pitch)
    M, b = standard_image_transform_3d(*n, 0.5, 0.5, 0.5)
    rng = np.random.default_rng(seed)
    y = rng.random((3, src.shape[0])).astype(np.float32)
    y[1] = np.where(y[1] > 0.5, y[1], 0.0)
    y[2] *= np.exp(rng.normal(0.0, 3.0, y.shape[1])).astype(np.float32)  # a wide dynamic range
    return dict(n=n, n_view=n_view, det=det, src=T(src), dst=T(dst), M=T(M), Minv=T(O.minv(M.numpy())), b=T(b),
                vol=T(rng.random(n).astype(np.float32)), y=T(y), y_np=y, Minv_np=O.minv(M.numpy()), b_np=b.numpy(),
                src_np=src.numpy(), dst_np=dst.numpy())


def opts_for(kind, c):
    from ct_laboratory_b200 import _native as N
    nv, nu = c["det"][1], c["det"][0]
    rule = N.VOXEL_CROSSING if kind.startswith("crossing") else N.VOXEL_MIDPOINT
    if kind.endswith("flat"):
        return N.flat_opts(voxel_rule=rule, block_threads=128)
    rows = 16 if kind.endswith("16") else 32
    return N.tiling(c["n_view"], nv, nu, nv * nu, nu, 1, tile_rows=rows, block_threads=128, voxel_rule=rule)


KINDS = ["midpoint-col32", "midpoint-col16", "midpoint-flat", "crossing-col32", "crossing-col16", "crossing-flat"]


@pytest.fixture(scope="module")
def cone():
    return case()


@pytest.mark.parametrize("kind", KINDS)
def test_fixed_adjoint_reproducible_and_matches_float(cone, kind):
    from ct_laboratory_b200 import _C
    from ct_laboratory_b200.tomography import back_project_3d_fixed_cuda
    c, opts = cone, opts_for(kind, cone)
    args = (c["src"], c["dst"], c["M"], c["b"], *c["n"])
    f1 = back_project_3d_fixed_cuda(c["y"], *args, tiling=opts, M_inv=c["Minv"])
    f2 = back_project_3d_fixed_cuda(c["y"], *args, tiling=opts, M_inv=c["Minv"])
    assert torch.equal(f1, f2)
    at = _C.back_project_3d_on_the_fly_cuda(c["y"], c["src"], c["dst"], c["Minv"], c["b"], *c["n"], tiling=opts)
    for i in range(3):
        assert rel_err(f1[i].cpu().numpy(), at[i].cpu().numpy()) < TOL_FLOAT, (kind, i)
        # alone or in a batch: the same bits (a per-sinogram scale, integer sums)
        alone = back_project_3d_fixed_cuda(c["y"][i].contiguous(), *args, tiling=opts, M_inv=c["Minv"])
        assert torch.equal(alone, f1[i]), (kind, i)
    if kind.startswith("midpoint"):
        ref = O.back_planesort(c["y_np"][0], c["Minv_np"], c["b_np"], c["src_np"], c["dst_np"], list(c["n"]))
        assert rel_err(f1[0].cpu().numpy(), ref) < TOL


def test_fixed_adjoint_identity(cone):
    from ct_laboratory_b200 import _C
    from ct_laboratory_b200.tomography import back_project_3d_fixed_cuda
    c = cone
    for kind in ("midpoint-col32", "crossing-col32"):
        opts = opts_for(kind, c)
        ax = _C.forward_project_3d_on_the_fly_cuda(c["vol"], c["src"], c["dst"], c["Minv"], c["b"], tiling=opts)[0]
        aty = back_project_3d_fixed_cuda(c["y"][0].contiguous(), c["src"], c["dst"], c["M"], c["b"], *c["n"],
                                         tiling=opts, M_inv=c["Minv"])
        lhs = float(ax.double() @ c["y"][0].double())
        rhs = float((c["vol"].double() * aty.double()).sum())
        assert abs(lhs - rhs) <= 1e-6 * abs(lhs), kind


def test_fixed_adjoint_zeros_accumulate_nonfinite_and_workspace(cone):
    from ct_laboratory_b200.tomography import back_project_3d_fixed_cuda, fixed_workspace_bytes
    c = cone
    args = (c["src"], c["dst"], c["M"], c["b"], *c["n"])
    opts = opts_for("midpoint-col32", c)
    z = back_project_3d_fixed_cuda(torch.zeros_like(c["y"][:1]), *args, tiling=opts)
    assert int(torch.count_nonzero(z)) == 0
    base = torch.full((1, *c["n"]), 0.25, device=DEV)
    acc = back_project_3d_fixed_cuda(c["y"][:1].contiguous(), *args, tiling=opts, out=base.clone(), accumulate=True)
    plain = back_project_3d_fixed_cuda(c["y"][:1].contiguous(), *args, tiling=opts)
    assert torch.equal(acc, plain + 0.25)
    # a sinogram holding NaN or inf gives a NaN volume; its batch-mates are untouched
    for bad in (float("nan"), float("inf")):
        y = c["y"][:2].clone()
        y[1, 7] = bad
        out = back_project_3d_fixed_cuda(y, *args, tiling=opts)
        assert bool(torch.isnan(out[1]).all())
        assert torch.equal(out[0], back_project_3d_fixed_cuda(c["y"][0].contiguous(), *args, tiling=opts))
    need = fixed_workspace_bytes(2, *c["n"])
    assert need >= 2 * 8 * int(np.prod(c["n"]))
    small = torch.empty(need - 256, dtype=torch.uint8, device=DEV)
    with pytest.raises(RuntimeError):
        back_project_3d_fixed_cuda(c["y"][:2].contiguous(), *args, tiling=opts, workspace=small)
    ws = torch.empty(need, dtype=torch.uint8, device=DEV)
    a = back_project_3d_fixed_cuda(c["y"][:2].contiguous(), *args, tiling=opts, workspace=ws)
    b = back_project_3d_fixed_cuda(c["y"][:2].contiguous(), *args, tiling=opts, workspace=ws)
    assert torch.equal(a, b)


@pytest.mark.parametrize("rule", [0, 1])
def test_fixed_module_backward(rule):
    """deterministic_adjoint=True: back_project and the autograd backward take
    the fixed-point scatter of the forward's own walk; both bitwise stable."""
    from ct_laboratory_b200 import ConeBeam3DProjector
    kw = dict(n_x=24, n_y=20, n_z=16, n_view=6, det_nx=32, det_ny=24, sid=100.0, sdd=150.0, det_spacing=0.8,
              voxel_size=0.5, device=torch.device(DEV), voxel_rule=rule)
    p = ConeBeam3DProjector(**kw, deterministic_adjoint=True)
    q = ConeBeam3DProjector(**kw)
    assert p.adjoint_mode == "fixed" and p.panels is None
    x = torch.rand(24, 20, 16, device=DEV, requires_grad=True)
    w = torch.rand(p.src.shape[0], device=DEV)
    (p(x) * w).sum().backward()
    g = x.grad.clone()
    x.grad = None
    (p(x) * w).sum().backward()
    assert torch.equal(g, x.grad)
    assert torch.equal(g, p.back_project(w))
    assert rel_err(g.cpu().numpy(), q.back_project(w).cpu().numpy()) < TOL_FLOAT


def test_fixed_adjoint_without_rays_and_host_errors():
    """No rays: the volume comes out zero (accumulate leaves it as it was);
    a workspace that is too small or misaligned, a batch outside [1, 65535]
    and a deterministic 2-D ScanBatch are refused on the host."""
    from ct_laboratory_b200 import FanBeam2DProjector
    from ct_laboratory_b200 import _native as N
    from ct_laboratory_b200.batched import ScanBatch
    n = (8, 6, 4)
    Mi = torch.eye(3, device=DEV).contiguous()
    b = torch.zeros(3, device=DEV)
    need = N.lib.ctlab_back_project_3d_fixed_workspace_bytes(1, *n)
    ws = torch.empty(need + 256, dtype=torch.uint8, device=DEV)
    out = torch.full((1, *n), 7.0, device=DEV)
    stream = N.stream_of(out)
    for acc, want in ((1, 7.0), (0, 0.0)):
        N.call("ctlab_back_project_3d_fixed", None, 1, 0, None, None, N.ptr(Mi), N.ptr(b), *n, N.ptr(out), acc,
               None, None, -1, N.ptr(ws), need, stream)
        torch.cuda.synchronize()
        assert bool((out == want).all())
    assert N.lib.ctlab_back_project_3d_fixed_workspace_bytes(0, *n) < 0
    rc = N.lib.ctlab_back_project_3d_fixed(None, 1, 0, None, None, N.ptr(Mi), N.ptr(b), *n, N.ptr(out), 0, None,
                                           None, -1, N.ptr(ws), need - 8, stream)
    assert rc != 0 and b"workspace" in N.lib.ctlab_last_error()
    odd = ws[8:]  # 8 bytes past a 256-byte boundary
    rc = N.lib.ctlab_back_project_3d_fixed(None, 1, 0, None, None, N.ptr(Mi), N.ptr(b), *n, N.ptr(out), 0, None,
                                           None, -1, N.ptr(odd), need, stream)
    assert rc != 0
    rc = N.lib.ctlab_back_project_3d_fixed(None, 0, 0, None, None, N.ptr(Mi), N.ptr(b), *n, N.ptr(out), 0, None,
                                           None, -1, N.ptr(ws), need, stream)
    assert rc != 0 and b"batch" in N.lib.ctlab_last_error()
    fan = FanBeam2DProjector(16, 16, n_view=4, n_det=20, sid=100.0, sdd=150.0, det_spacing=1.0, pixel_size=1.0,
                             device=torch.device(DEV))
    with pytest.raises(ValueError):
        ScanBatch([fan], deterministic_adjoint=True)
