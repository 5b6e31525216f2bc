"""Spectral CT system: a projector composed with an X-ray system model.

Mirrors the reference's CTSystem (physics/ct_system/ct_system.py:19-96):

    basis volumes [n_materials, nx, ny, nz]
        --A-->  basis line integrals x_basis [n_rays, n_materials]
        --xray_system-->  detector statistics

``xray_system`` is any object with the reference XraySystem's interface
(``__call__`` / ``forward_stats`` / ``log_prob`` / ``sample`` /
``decompose_basis`` on x_basis, and ``basis_materials.n_materials``); the
reference's own XraySystem is pure PyTorch and plugs in unchanged.  The
projector side runs on the B200 kernels: where the reference projects the
basis volumes one material at a time, here all materials go through the
projector as one batch of volumes (one forward launch, one adjoint launch),
and the projection stays differentiable through the projector's autograd
Function.
"""
from __future__ import annotations

from torch import nn

__all__ = ["CTSystem"]


class CTSystem(nn.Module):
    def __init__(self, projector, xray_system):
        super().__init__()
        for required in ("forward_project", "back_project"):
            if not hasattr(projector, required):
                raise TypeError(f"projector must expose {required!r}; got {type(projector).__name__}")
        self.projector = projector
        self.xray_system = xray_system

    @property
    def n_materials(self):
        return self.xray_system.basis_materials.n_materials

    def project_basis(self, basis_volumes):
        """[n_materials, nx, ny, nz] (or one volume) -> x_basis [n_rays, n_materials]."""
        if basis_volumes.dim() == 3:
            basis_volumes = basis_volumes.unsqueeze(0)
        sino = self.projector.forward_project(basis_volumes.contiguous())  # [n_materials, n_rays]
        return sino.reshape(basis_volumes.shape[0], -1).t()

    def back_project_basis(self, x_basis):
        """Adjoint of project_basis: [n_rays, n_materials] -> [n_materials, nx, ny, nz]."""
        vols = self.projector.back_project(x_basis.t().contiguous())
        return vols if vols.dim() == 4 else vols.unsqueeze(0)

    def forward_stats(self, basis_volumes, **kwargs):
        return self.xray_system.forward_stats(self.project_basis(basis_volumes), **kwargs)

    def forward(self, basis_volumes, **kwargs):
        return self.xray_system(self.project_basis(basis_volumes), **kwargs)

    def log_prob(self, y_obs, basis_volumes, **kwargs):
        return self.xray_system.log_prob(y_obs, self.project_basis(basis_volumes), **kwargs)

    def sample(self, basis_volumes, **kwargs):
        return self.xray_system.sample(self.project_basis(basis_volumes), **kwargs)

    def decompose_basis(self, y_obs, **kwargs):
        return self.xray_system.decompose_basis(y_obs, **kwargs)
