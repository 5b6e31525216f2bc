"""Subset projectors: the reference's ct_projector_3d_subsets area on the B200
kernels.

Same classes, constructors, attributes and results as the reference
(tomography/ct_projector_3d_subsets.py:9-276):

``SubsetProjector``         resolves the innermost CTProjector3DModule
                            (``core_module``) of a projector stack and builds
                            modules over subsets of its rays;
``OrderedSubsetProjector``  the rays in ``n_subsets`` contiguous blocks of at
                            most ``max_subset_size`` with their intersection
                            tables: sliced from the core's loaded tables,
                            loaded from the per-subset cache files in
                            ``cache_dir`` (the reference's file names), or
                            computed and saved there;
``RandomSubsetProjector``   a random subset of the rays (``torch.randperm``
                            under ``torch.manual_seed(seed)``, as the
                            reference draws it).

One difference, not in results: the reference always projects through
per-subset tables, because its table-free kernel is quadratic in the planes
per ray.  Here, when the core has no tables loaded and no ``cache_dir`` is
given (``use_tables=None``), the ordered projector projects all rays in one
on-the-fly launch instead of building tables subset by subset: the
subsets only ever bounded table memory.  ``use_tables=True`` keeps the
reference's table path (compressed tables quantise the plane parameters, so
the two differ by the compression error, ~1e-4 relative).
"""
from __future__ import annotations

import os
import time

import numpy as np
import torch
from torch import nn

from .ct_projector_3d_module import CTProjector3DModule, precompute_tvals_stitched

__all__ = ["SubsetProjector", "OrderedSubsetProjector", "RandomSubsetProjector"]


class SubsetProjector(nn.Module):
    """Base of the subset projectors (reference :9-57)."""

    def __init__(self, base_projector, subset_size, precomputed_intersections=False, verbose=False):
        super().__init__()
        self.base_projector = base_projector
        self.subset_size = subset_size
        self.precomputed_intersections = precomputed_intersections
        self.verbose = verbose
        core = base_projector
        while hasattr(core, "base_projector") and not isinstance(core, CTProjector3DModule):
            core = core.base_projector
        if not isinstance(core, CTProjector3DModule):
            raise ValueError("base_projector must eventually be a CTProjector3DModule")
        self.core_module = core
        self.n_total_rays_core = core.src.shape[0]
        device = core.src.device
        self.device = torch.device("cuda") if device.type == "cpu" and torch.cuda.is_available() else device
        self.n_x, self.n_y, self.n_z = core.n_x, core.n_y, core.n_z
        self.M, self.b = core.M, core.b
        self.backend = core.backend

    def _get_subset_module(self, indices):
        """A CTProjector3DModule over the core rays `indices` (on the fly)."""
        core = self.core_module
        idx = indices.to(core.src.device)
        return CTProjector3DModule(n_x=self.n_x, n_y=self.n_y, n_z=self.n_z, M=self.M.to(self.device),
                                   b=self.b.to(self.device), src=core.src[idx].to(self.device),
                                   dst=core.dst[idx].to(self.device), backend=self.backend, device=self.device,
                                   precomputed_intersections=self.precomputed_intersections)

    def _run_forward(self, module, volume):
        return module.forward(volume)

    def _run_backward(self, module, sinogram):
        return module.back_project(sinogram)


class OrderedSubsetProjector(SubsetProjector):
    """Rays in contiguous blocks with their tables (reference :59-229)."""

    def __init__(self, base_projector, max_subset_size=1_000_000, cache_dir=None, verbose=False, use_tables=None):
        super().__init__(base_projector, max_subset_size, precomputed_intersections=True, verbose=verbose)
        self.cache_dir = cache_dir
        self.n_subsets = int(np.ceil(self.n_total_rays_core / self.subset_size))
        self.subset_boundaries = np.linspace(0, self.n_total_rays_core, self.n_subsets + 1, dtype=int)
        self.last_precompute_time = 0.0
        self.last_projection_time = 0.0
        core = self.core_module
        has_tables = core.tvals_uint16 is not None or core.tvals_full is not None
        self.use_tables = bool(has_tables or cache_dir is not None) if use_tables is None else bool(use_tables)
        self.persistent_projector = None
        if not self.use_tables:
            self.persistent_projector = core
        elif self.n_subsets == 1:
            t0 = time.time()
            self.persistent_projector = self._get_cached_subset_projector(0)
            self.persistent_projector.to(self.device)
            self.last_precompute_time = time.time() - t0

    # -- caching (file names as the reference's, :85-97) ----------------------
    def _get_subset_cache_path(self, j):
        if self.cache_dir is None:
            return None
        start_ray, end_ray = int(self.subset_boundaries[j]), int(self.subset_boundaries[j + 1])
        fname = f"tvals_subset{j:04d}_rays{start_ray}-{end_ray}_nx{self.n_x}_ny{self.n_y}_nz{self.n_z}.pt"
        return os.path.join(self.cache_dir, fname)

    def _get_cached_subset_projector(self, j):
        """Module for subset j with its tables: sliced from the core's loaded
        tables, else loaded from / computed into the cache (reference :99-150)."""
        s, e = int(self.subset_boundaries[j]), int(self.subset_boundaries[j + 1])
        core = self.core_module
        if core.tvals_uint16 is not None:
            sub = (core.tvals_uint16[s:e], core.tvals_start[s:e], core.tvals_scale[s:e])
        elif core.tvals_full is not None:
            sub = core.tvals_full[s:e]
        else:
            path = self._get_subset_cache_path(j)
            if path is not None and os.path.exists(path):
                if self.verbose:
                    print(f"  Loading subset {j} tvals: {path}", flush=True)
                sub = torch.load(path, map_location="cpu")
            else:
                if self.verbose:
                    print(f"  Computing subset {j} tvals ({e - s} rays)...", flush=True)
                sub = precompute_tvals_stitched(self.n_x, self.n_y, self.n_z, self.M, self.b, core.src[s:e],
                                                core.dst[s:e], device=self.device, verbose=self.verbose)
                if path is not None:
                    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
                    torch.save(sub, path)
        return CTProjector3DModule(n_x=self.n_x, n_y=self.n_y, n_z=self.n_z, M=self.M, b=self.b, src=core.src[s:e],
                                   dst=core.dst[s:e], backend=self.backend, device=self.device, tvals=sub)

    def forward(self, volume):
        self.last_precompute_time = self.last_projection_time = 0.0
        if self.persistent_projector is not None:
            t0 = time.time()
            res = self._run_forward(self.persistent_projector, volume)
            self.last_projection_time = time.time() - t0
            return res
        n = self.n_total_rays_core
        shape = (volume.shape[0], n) if volume.dim() == 4 else (n,)
        out = torch.zeros(shape, device=volume.device, dtype=volume.dtype)
        for j in range(self.n_subsets):
            s, e = int(self.subset_boundaries[j]), int(self.subset_boundaries[j + 1])
            t0 = time.time()
            sub = self._get_cached_subset_projector(j).to(volume.device)
            t1 = time.time()
            out[..., s:e] = self._run_forward(sub, volume)
            self.last_precompute_time += t1 - t0
            self.last_projection_time += time.time() - t1
            del sub
        return out

    def forward_project(self, volume):
        return self.forward(volume)

    def back_project(self, sinogram):
        self.last_precompute_time = self.last_projection_time = 0.0
        if self.persistent_projector is not None:
            t0 = time.time()
            res = self._run_backward(self.persistent_projector, sinogram)
            self.last_projection_time = time.time() - t0
            return res
        vol = None
        for j in range(self.n_subsets):
            s, e = int(self.subset_boundaries[j]), int(self.subset_boundaries[j + 1])
            t0 = time.time()
            sub = self._get_cached_subset_projector(j).to(sinogram.device)
            t1 = time.time()
            part = self._run_backward(sub, sinogram[..., s:e].contiguous())
            vol = part if vol is None else vol.add_(part)
            self.last_precompute_time += t1 - t0
            self.last_projection_time += time.time() - t1
            del sub
        return vol


class RandomSubsetProjector(SubsetProjector):
    """A random subset of the core rays (reference :231-276)."""

    def __init__(self, base_projector, subset_size=10000, precomputed_intersections=False, randomize_on_forward=False,
                 randomize_on_backward=False, seed=None, verbose=False):
        super().__init__(base_projector, subset_size, precomputed_intersections, verbose)
        self.randomize_on_forward = randomize_on_forward
        self.randomize_on_backward = randomize_on_backward
        self.seed = seed
        self.current_subset_module = None
        self.current_indices = None
        self.randomize_projector()

    def randomize_projector(self, subset_size=None, seed=None):
        if subset_size is not None:
            self.subset_size = subset_size
        if seed is not None:
            self.seed = seed
        if self.seed is not None:
            torch.manual_seed(self.seed)
        self.current_indices = torch.randperm(self.n_total_rays_core, device="cpu")[:self.subset_size]
        self.current_subset_module = None
        self.current_subset_module = self._get_subset_module(self.current_indices)

    def forward(self, volume):
        if self.randomize_on_forward:
            self.randomize_projector()
        return self._run_forward(self.current_subset_module, volume)

    def back_project(self, sinogram):
        if self.randomize_on_backward:
            self.randomize_projector()
        return self._run_backward(self.current_subset_module, sinogram)

    def forward_project(self, volume):
        return self.forward(volume)
