"""CTSystem (reference physics/ct_system/ct_system.py) on the B200
projector: the basis volumes projected as one batch equal the reference's
per-material loop, the basis adjoint is the transpose, and the spectral
log-likelihood differentiates into the basis volumes.  A two-channel
Beer-Lambert model stands in for the reference's XraySystem (same
interface; the physics itself is outside this build)."""
from types import SimpleNamespace

import pytest
import torch
from torch import nn

from conftest import rel_err

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")


class TwoChannelSystem(nn.Module):
    basis_materials = SimpleNamespace(n_materials=2)

    def __init__(self, I0=1e4):
        super().__init__()
        self.I0 = I0
        self.mu = torch.tensor([[0.20, 0.10], [0.15, 0.30]], device=DEV)  # [channel, material]

    def forward(self, x_basis):
        return self.I0 * torch.exp(-(x_basis @ self.mu.t()))

    def forward_stats(self, x_basis):
        m = self(x_basis)
        return m, m

    def log_prob(self, y, x_basis):
        return torch.distributions.Poisson(self(x_basis)).log_prob(y).sum()

    def sample(self, x_basis):
        return torch.poisson(self(x_basis))

    def decompose_basis(self, y):
        return -torch.log(y / self.I0) @ torch.linalg.inv(self.mu).t()


def test_ct_system_batches_materials_and_differentiates():
    from ct_laboratory_b200 import ConeBeam3DProjector
    from ct_laboratory_b200.ct_system import CTSystem
    p = ConeBeam3DProjector(20, 18, 14, n_view=8, det_nx=28, det_ny=20, sid=100.0, sdd=150.0, det_spacing=0.8,
                            voxel_size=0.5, voxel_rule=1, device=DEV)
    sysm = CTSystem(p, TwoChannelSystem())
    assert sysm.n_materials == 2
    g = torch.Generator(device=DEV).manual_seed(0)
    basis = 0.05 * torch.rand(2, 20, 18, 14, generator=g, device=DEV)
    xb = sysm.project_basis(basis)
    loop = torch.stack([p.forward_project(v).reshape(-1) for v in basis], dim=1)
    assert xb.shape == (p.src.shape[0], 2) and torch.equal(xb, loop)
    r = torch.rand(p.src.shape[0], 2, generator=g, device=DEV)
    bt = sysm.back_project_basis(r)
    loop_b = torch.stack([p.back_project(r[:, m].contiguous()) for m in range(2)], dim=0)
    assert bt.shape == basis.shape and rel_err(bt.cpu().numpy(), loop_b.cpu().numpy()) < 1e-5
    lhs, rhs = float((xb.double() * r.double()).sum()), float((basis.double() * bt.double()).sum())
    assert abs(lhs - rhs) < 1e-5 * abs(lhs)
    y = sysm.sample(basis)
    v = basis.clone().requires_grad_(True)
    sysm.log_prob(y, v).backward()
    # log p = sum y log m - m with m = I0 exp(-x mu^T): d log p / dx = (m - y) mu, then A^T per material
    with torch.no_grad():
        mean = sysm(basis)
        dx = (mean - y) @ sysm.xray_system.mu  # [n_rays, n_materials]
        want = sysm.back_project_basis(dx)
    assert rel_err(v.grad.cpu().numpy(), want.cpu().numpy()) < 1e-4
