"""CTProjector2DModule: the reference's 2-D projector nn.Module, B200 backed.

Same constructor and methods as the reference
(tomography/ct_projector_2d_module.py:11-65): ``forward`` (differentiable),
``forward_project``, ``back_project`` and a ``tvals`` table.  The reference
always builds the [n_ray, (R+1)+(C+1)] table in __init__ and projects from
it.  Here the default projects with the table-free Siddon kernel, which
evaluates the same plane parameters on the fly (no table memory, one pass);
``precomputed_intersections=True`` builds the table on the GPU and uses the
table kernels, whose per-segment arithmetic is the reference's.  ``tvals``
is available either way (built on first access when not precomputed).

``deterministic_adjoint=True`` (with a detector-line table ``panels``, from
``panels_from_lines_2d``; the fan-beam and uniform StaticCT classes build it)
makes ``back_project`` and the autograd backward gather per pixel instead of
scattering with atomics: bitwise reproducible, the exact transpose of the
crossing-rule forward, used when no table is loaded.
"""
from __future__ import annotations

import torch

from ._common import InverseCache, require_cuda
from .ct_projector_2d_autograd import CTProjector2DFunction
from .ct_projector_2d_cuda import back_project_2d_cuda, compute_intersections_2d_cuda, forward_project_2d_cuda
from .gather import back_project_2d_gather_cuda, embed_2d_geometry

__all__ = ["CTProjector2DModule"]


class CTProjector2DModule(torch.nn.Module):
    def __init__(self, n_row, n_col, M, b, src, dst, backend="cuda", precomputed_intersections=False,
                 ray_tiling=None, panels=None, deterministic_adjoint=False):
        super().__init__()
        self.deterministic_adjoint = bool(deterministic_adjoint)
        if self.deterministic_adjoint and panels is None:
            raise ValueError("deterministic_adjoint needs a detector-line table (panels_from_lines_2d)")
        self.panels = panels
        self._geom3 = None
        self.backend = backend
        self.n_row, self.n_col = int(n_row), int(n_col)
        self.ray_tiling = ray_tiling
        self._minv = InverseCache()
        # the kernels read raw pointers: keep contiguous float32 copies
        f32 = lambda t: t.to(torch.float32).contiguous()  # noqa: E731
        self.register_buffer("M", f32(M))
        self.register_buffer("b", f32(b))
        self.register_buffer("src", f32(src))
        self.register_buffer("dst", f32(dst))
        self.precomputed_intersections = bool(precomputed_intersections)
        self._tvals = None
        if self.precomputed_intersections:
            require_cuda(src, dst, M, b, what="geometry for precomputed intersections")
            self._tvals = compute_intersections_2d_cuda(self.n_row, self.n_col, self.M, self.b, self.src, self.dst,
                                                        M_inv=self.M_inv)

    @property
    def M_inv(self):
        return self._minv.get(self.M)

    @property
    def tvals(self):
        if self._tvals is None or self._tvals.device != self.src.device:
            self._tvals = compute_intersections_2d_cuda(self.n_row, self.n_col, self.M, self.b, self.src, self.dst,
                                                        M_inv=self.M_inv)
        return self._tvals

    def _table(self):
        return self.tvals if self.precomputed_intersections else None

    def _gather(self):
        """The deterministic adjoint y -> A^T y, or None for the atomic one."""
        if not self.deterministic_adjoint or self._table() is not None:
            return None
        if self._geom3 is None or self._geom3[0].device != self.src.device:
            self._geom3 = embed_2d_geometry(self.src, self.dst, self.M, self.b)
        panels = self.panels.to(self.src.device)
        return lambda y: back_project_2d_gather_cuda(y, self._geom3, self.n_row, self.n_col, panels)

    def forward_project(self, volume):
        require_cuda(volume, what="image")
        return forward_project_2d_cuda(volume.contiguous(), self._table(), self.M, self.b, self.src, self.dst,
                                       tiling=self.ray_tiling, M_inv=self.M_inv)

    def back_project(self, sinogram):
        require_cuda(sinogram, what="sinogram")
        gather = self._gather()
        if gather is not None:
            return gather(sinogram.contiguous())
        return back_project_2d_cuda(sinogram.contiguous(), self._table(), self.M, self.b, self.src, self.dst,
                                    self.n_row, self.n_col, tiling=self.ray_tiling, M_inv=self.M_inv)

    def forward(self, image):
        require_cuda(image, what="image")
        return CTProjector2DFunction.apply(image, self._table(), self.M, self.b, self.src, self.dst, self.backend,
                                           self.ray_tiling, self.M_inv, self._gather())
