"""The reference-facing API on the GPU: modules, autograd, finite
differences, tvals save/load, precompute.  Mirrors the reference's module
tests (python_examples/test_ct_projector_{2d,3d}_module.py: forward, sum,
backward, grad present) with numeric checks added."""
import os

import numpy as np
import pytest
import torch

from conftest import load_golden, rel_err
from oracle import oracle as O

pytestmark = pytest.mark.gpu
DEV = "cuda"


def small_cone(**kw):
    from ct_laboratory_b200 import ConeBeam3DProjector
    args = dict(n_x=32, n_y=28, n_z=24, n_view=16, det_nx=40, det_ny=32, sid=100.0, sdd=150.0, det_spacing=0.8,
                voxel_size=0.5)
    args.update(kw)
    return ConeBeam3DProjector(**args, device=torch.device(DEV))


def test_module_smoke_like_reference():
    """test_ct_projector_3d_module.py:17-63: 8^3 volume, 2 rays, forward,
    sum, backward; plus 2-D (test_ct_projector_2d_module.py:17-65)."""
    from ct_laboratory_b200 import CTProjector2DModule, CTProjector3DModule
    M, b = torch.eye(3, device=DEV), torch.zeros(3, device=DEV)
    src = torch.tensor([[-10.0, 3.5, 3.5], [3.2, -10.0, 4.1]], device=DEV)
    dst = torch.tensor([[10.0, 3.5, 3.5], [3.7, 10.0, 2.0]], device=DEV)
    p = CTProjector3DModule(8, 8, 8, M, b, src, dst, device=torch.device(DEV))
    vol = torch.rand(8, 8, 8, device=DEV, requires_grad=True)
    sino = p(vol)
    assert sino.shape == (2,)
    sino.sum().backward()
    assert vol.grad is not None and vol.grad.shape == vol.shape
    assert torch.allclose(vol.grad, p.back_project(torch.ones(2, device=DEV)))
    M2, b2 = torch.eye(2, device=DEV), torch.zeros(2, device=DEV)
    s2 = torch.tensor([[-5.0, 2.5], [2.0, -5.0], [-5.0, -5.0]], device=DEV)
    d2 = torch.tensor([[20.0, 2.5], [2.0, 20.0], [20.0, 20.0]], device=DEV)
    for pre in (False, True):
        p2 = CTProjector2DModule(16, 16, M2, b2, s2, d2, precomputed_intersections=pre)
        img = torch.rand(16, 16, device=DEV, requires_grad=True)
        out = p2(img)
        out.sum().backward()
        assert out.shape == (3,) and img.grad.shape == (16, 16)


def test_finite_differences_16_voxels():
    """Gradient of 0.5||Ax - y||^2 against central differences (step 1e-3,
    16 seeded voxels), the check of the MAP configuration."""
    p = small_cone()
    g = torch.Generator(device="cpu").manual_seed(0)
    x = (0.01 * torch.rand(32, 28, 24, generator=g)).to(DEV)
    y = p(x).detach() + 0.05 * torch.rand(p.src.shape[0], generator=g).to(DEV)

    def loss(v):
        r = (p(v) - y).double()
        return 0.5 * float((r * r).sum())

    xr = x.clone().requires_grad_(True)
    r = p(xr) - y
    (0.5 * (r * r).sum()).backward()
    grad = xr.grad.double().cpu()
    idx = torch.randint(0, x.numel(), (16,), generator=g)
    # restrict to voxels some ray sees
    seen = p.back_project(torch.ones_like(y)).flatten().cpu() > 0
    idx = torch.nonzero(seen).flatten()[torch.randint(0, int(seen.sum()), (16,), generator=g)]
    h = 1e-3
    for i in idx.tolist():
        e = torch.zeros(x.numel(), device=DEV)
        e[i] = h
        e = e.view_as(x)
        fd = (loss(x + e) - loss(x - e)) / (2 * h)
        assert abs(fd - float(grad.flatten()[i])) <= 2e-3 * max(abs(fd), 1e-3), (i, fd, float(grad.flatten()[i]))


def test_batched_volume_and_sinogram():
    p = small_cone(n_view=4)
    x = torch.rand(3, 32, 28, 24, device=DEV)
    s = p(x)
    assert s.shape == (3, p.src.shape[0])
    for k in range(3):
        assert torch.allclose(s[k], p(x[k]), rtol=0, atol=0)
    bp = p.back_project(s)
    assert bp.shape == (3, 32, 28, 24)
    assert torch.allclose(bp[1], p.back_project(s[1]), rtol=1e-5, atol=1e-5)


def test_cone_module_matches_oracle_and_tiling_is_transparent():
    from ct_laboratory_b200 import CTProjector3DModule
    p = small_cone()
    x = torch.rand(32, 28, 24, device=DEV)
    tiled = p(x)
    flat = CTProjector3DModule(32, 28, 24, p.M, p.b, p.src, p.dst, device=torch.device(DEV))(x)
    assert torch.equal(tiled, flat)  # same arithmetic per ray, only the launch shape differs
    ref = O.fwd_planesort(x.cpu().numpy(), O.minv(p.M.cpu().numpy()), p.b.cpu().numpy(), p.src.cpu().numpy(),
                          p.dst.cpu().numpy())
    assert rel_err(tiled.cpu().numpy(), ref) < 1e-5


def test_precomputed_compressed_module_and_tvals_io(tmp_path):
    from ct_laboratory_b200 import CTProjector3DModule, precompute_tvals_stitched
    g = load_golden("cone3d")
    M, b, src, dst = (torch.as_tensor(g[k]).to(DEV) for k in ("M", "b", "src", "dst"))
    p = CTProjector3DModule(14, 12, 10, M, b, src, dst, device=torch.device(DEV), precomputed_intersections=True)
    # the module trims all-inf columns and encodes with the torch encoder:
    # identical to encoding the (trimmed) reference table
    fin_cols = np.isfinite(g["tvals"]).any(axis=0)
    K = int(np.argmin(fin_cols)) if not fin_cols.all() else g["tvals"].shape[1]
    u_ref, s_ref, c_ref = O.compress_torch(g["tvals"][:, :K], g["src"], g["dst"], float(g["voxel_diag"]))
    assert np.array_equal(p.tvals_uint16.cpu().numpy().view(np.uint16), u_ref)
    assert np.array_equal(p.tvals_start.cpu().numpy(), s_ref)
    vol = torch.as_tensor(g["vol"]).to(DEV)
    out = p(vol).cpu().numpy()
    ref = O.fwd_comp_cuda(g["vol"], u_ref, s_ref, c_ref, g["Minv"], g["b"], g["src"], g["dst"])
    assert rel_err(out, ref) < 1e-5
    path = os.path.join(tmp_path, "tv.pt")
    p.save_tvals(path)
    d = torch.load(path)
    assert set(d) == {"tvals_uint16", "tvals_start", "tvals_scale", "tvals_full", "n_x", "n_y", "n_z", "n_ray"}
    q = CTProjector3DModule(14, 12, 10, M, b, src, dst, device=torch.device(DEV))
    q.load_tvals(path)
    assert torch.equal(q(vol), p(vol))
    # stitched precompute with the CUDA encoder equals the restated reference kernel
    t16, st, sc = precompute_tvals_stitched(14, 12, 10, M.cpu(), b.cpu(), src.cpu(), dst.cpu(), chunk_size=100,
                                            verbose=False)
    u_o, st_o, sc_o = O.compress_cuda(g["tvals"], g["src"], g["dst"], float(g["voxel_diag"]))
    assert np.array_equal(t16.numpy().view(np.uint16), u_o) and np.array_equal(st.numpy(), st_o)
    full = precompute_tvals_stitched(14, 12, 10, M.cpu(), b.cpu(), src.cpu(), dst.cpu(), chunk_size=77,
                                     verbose=False, use_compression=False)
    assert np.array_equal(full.numpy(), g["tvals"])


def test_fanbeam_and_static2d_modules():
    from ct_laboratory_b200 import FanBeam2DProjector
    p = FanBeam2DProjector(40, 36, n_view=10, n_det=48, sid=60.0, sdd=100.0, det_spacing=1.1, pixel_size=0.9,
                           device=torch.device(DEV))
    g = load_golden("fan2d")
    img = torch.as_tensor(g["img"]).to(DEV)
    assert rel_err(p(img).cpu().numpy(), g["fwd"]) < 1e-5
    assert rel_err(p.back_project(torch.as_tensor(g["y"]).to(DEV)).cpu().numpy(), g["back"]) < 1e-5
    assert np.array_equal(p.tvals.cpu().numpy(), g["tvals"])


@pytest.mark.parametrize("name", ["cone3d", "affine3d", "static3d"])
def test_autograd_gradient_matches_reference_gradient(name):
    """d/dvol sum(y * A vol) through our autograd Function equals the
    reference's own A^T y (its torch path, stored in the golden fixture), the
    gradient its CTProjector3DFunction backward returns
    (ct_projector_3d_autograd.py:160-170).  Tolerance: the spread between the
    reference's torch and CUDA paths, 5e-5."""
    from ct_laboratory_b200 import CTProjector3DModule
    g = load_golden(name)
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a)).to(DEV, torch.float32)  # noqa: E731
    d = [int(v) for v in g["dims"]]
    p = CTProjector3DModule(*d, T(g["M"]), T(g["b"]), T(g["src"]), T(g["dst"]), device=torch.device(DEV))
    vol = T(g["vol"]).requires_grad_(True)
    (p(vol) * T(g["y"])).sum().backward()
    assert rel_err(vol.grad.cpu().numpy(), g["back"]) < 5e-5
