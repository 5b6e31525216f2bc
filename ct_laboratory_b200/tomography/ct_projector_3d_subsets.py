"""Subset projectors: the reference's ct_projector_3d_subsets area on the B200
kernels.

Same classes, constructor arguments, attributes and results as the reference
(tomography/ct_projector_3d_subsets.py:9-276):

``SubsetProjector``         finds the innermost CTProjector3DModule
                            (``core_module``) under a stack of wrappers;
``OrderedSubsetProjector``  the rays in ``n_subsets`` contiguous ranges of at
                            most ``max_subset_size``, each projected through
                            its intersection table: a slice of the core's
                            loaded table, the per-subset cache file in
                            ``cache_dir`` (the reference's file names), or one
                            computed on the GPU and saved there;
``RandomSubsetProjector``   a random subset of the rays, drawn as the
                            reference draws it (``torch.randperm`` under
                            ``torch.manual_seed(seed)``).

How they run here.  The reference builds a CTProjector3DModule per subset
on every call.  Here a subset is a ray range (or an index list) handed to the
projector's autograd Function directly: the ordered projector projects
src[s:e] / dst[s:e] with the range's table and concatenates the ranges'
sinograms (the adjoint accumulates their volumes), keeping the tables of all
ranges resident when they came from the core or fit the `keep_tables`
budget; the random projector gathers its rays into reused device buffers and
projects them on the fly.  With no tables loaded and no ``cache_dir``
(``use_tables=None``) the ordered projector projects all rays in one
on-the-fly launch: the reference's ranges only ever bounded table memory, and
its table-free kernel is quadratic in the planes per ray while this one is
not.  ``use_tables=True`` keeps the table path (compressed tables quantise the
plane parameters, so the two differ by the compression error, ~1e-4
relative).
"""
from __future__ import annotations

import os
import time

import numpy as np
import torch
from torch import nn

from .. import _native as N
from .ct_projector_3d_autograd import CTProjector3DFunction
from .ct_projector_3d_cuda import back_project_3d_cuda
from .ct_projector_3d_module import CTProjector3DModule, precompute_tvals_stitched

__all__ = ["SubsetProjector", "OrderedSubsetProjector", "RandomSubsetProjector"]


def _innermost(projector):
    """The CTProjector3DModule at the bottom of a chain of `base_projector`s."""
    node = projector
    while not isinstance(node, CTProjector3DModule):
        node = getattr(node, "base_projector", None)
        if node is None:
            raise ValueError("base_projector must eventually be a CTProjector3DModule")
    return node


def _table_bytes(t):
    if t is None:
        return 0
    if isinstance(t, (tuple, list)):
        return sum(x.numel() * x.element_size() for x in t)
    return t.numel() * t.element_size()


def _on(t, device):
    if isinstance(t, (tuple, list)):
        return tuple(x.to(device) for x in t)
    return t.to(device)


def _parts(table):
    """(t_main, t_start, t_scale) of a float or compressed table."""
    if isinstance(table, (tuple, list)):
        return tuple(table)
    return table, None, None


class SubsetProjector(nn.Module):
    """Base of the subset projectors (reference :9-57): the core module, its
    grid, affine and backend, and the device the subsets run on (the GPU
    when the core sits on the host)."""

    def __init__(self, base_projector, subset_size, precomputed_intersections=False, verbose=False):
        super().__init__()
        self.base_projector = base_projector
        self.subset_size = subset_size
        self.precomputed_intersections = precomputed_intersections
        self.verbose = verbose
        self.core_module = _innermost(base_projector)
        core = self.core_module
        self.n_total_rays_core = core.src.shape[0]
        here = core.src.device
        self.device = torch.device("cuda") if here.type == "cpu" and torch.cuda.is_available() else here
        self.n_x, self.n_y, self.n_z = core.n_x, core.n_y, core.n_z
        self.M, self.b = core.M, core.b
        self.backend = core.backend

    def _get_subset_module(self, indices):
        """A CTProjector3DModule over the core rays `indices`."""
        core = self.core_module
        pick = indices.to(core.src.device)
        return CTProjector3DModule(n_x=self.n_x, n_y=self.n_y, n_z=self.n_z, M=self.M.to(self.device),
                                   b=self.b.to(self.device), src=core.src.index_select(0, pick).to(self.device),
                                   dst=core.dst.index_select(0, pick).to(self.device), backend=self.backend,
                                   device=self.device, precomputed_intersections=self.precomputed_intersections)

    def _run_forward(self, module, volume):
        return module.forward(volume)

    def _run_backward(self, module, sinogram):
        return module.back_project(sinogram)

    def _geometry(self, device):
        core = self.core_module
        return core.src.to(device), core.dst.to(device), core.M.to(device), core.b.to(device)


class OrderedSubsetProjector(SubsetProjector):
    """Rays in contiguous ranges, each with its table (reference :59-229).

    ``keep_tables``: bytes of tables loaded from or written to ``cache_dir``
    that may stay resident between calls (default 8 GiB); ranges beyond it
    are reloaded on every call, as the reference does with all of them."""

    def __init__(self, base_projector, max_subset_size=1_000_000, cache_dir=None, verbose=False, use_tables=None,
                 keep_tables=8 << 30):
        super().__init__(base_projector, max_subset_size, precomputed_intersections=True, verbose=verbose)
        self.cache_dir = cache_dir
        self.n_subsets = int(np.ceil(self.n_total_rays_core / self.subset_size))
        self.subset_boundaries = np.linspace(0, self.n_total_rays_core, self.n_subsets + 1, dtype=int)
        self.last_precompute_time = 0.0
        self.last_projection_time = 0.0
        self.keep_tables = int(keep_tables)
        core = self.core_module
        core_tables = core.tvals_uint16 is not None or core.tvals_full is not None
        self.use_tables = bool(core_tables or cache_dir is not None) if use_tables is None else bool(use_tables)
        self._tables = {}  # range j -> resident table
        # the reference keeps one module when a single range holds every ray;
        # here the table path needs no module, the table-free path is the core
        self.persistent_projector = None if self.use_tables else core
        if self.use_tables and self.n_subsets == 1:
            t0 = time.time()
            self._tables[0] = _on(self._table_of(0), self.device)
            self.last_precompute_time = time.time() - t0

    def _range(self, j):
        return int(self.subset_boundaries[j]), int(self.subset_boundaries[j + 1])

    # -- the reference's per-range cache files (:85-97) --------------------------
    def _get_subset_cache_path(self, j):
        if self.cache_dir is None:
            return None
        s, e = self._range(j)
        return os.path.join(self.cache_dir, f"tvals_subset{j:04d}_rays{s}-{e}_nx{self.n_x}_ny{self.n_y}_nz{self.n_z}.pt")

    def _table_of(self, j):
        """Range j's table: from the core's loaded table, else the cache
        file, else built on the GPU (and written to the cache)."""
        s, e = self._range(j)
        core = self.core_module
        if core.tvals_uint16 is not None:
            return core.tvals_uint16[s:e], core.tvals_start[s:e], core.tvals_scale[s:e]
        if core.tvals_full is not None:
            return core.tvals_full[s:e]
        path = self._get_subset_cache_path(j)
        if path is not None and os.path.exists(path):
            if self.verbose:
                print(f"  Loading subset {j} tvals: {path}", flush=True)
            return torch.load(path, map_location="cpu")
        if self.verbose:
            print(f"  Computing subset {j} tvals ({e - s} rays)...", flush=True)
        table = precompute_tvals_stitched(self.n_x, self.n_y, self.n_z, self.M, self.b, core.src[s:e], core.dst[s:e],
                                          device=self.device, verbose=self.verbose)
        if path is not None:
            os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
            torch.save(table, path)
        return table

    def _resident_table(self, j, device):
        table = self._tables.get(j)
        if table is None:
            table = _on(self._table_of(j), device)
            held = sum(_table_bytes(t) for t in self._tables.values())
            from_core = self.core_module.tvals_uint16 is not None or self.core_module.tvals_full is not None
            if from_core or held + _table_bytes(table) <= self.keep_tables:
                self._tables[j] = table
        return table

    def _ranges(self, device):
        """(s, e, table) per range, with the timing split the reference keeps."""
        for j in range(self.n_subsets):
            t0 = time.time()
            table = self._resident_table(j, device)
            self.last_precompute_time += time.time() - t0
            s, e = self._range(j)
            yield s, e, table

    def forward(self, volume):
        self.last_precompute_time = self.last_projection_time = 0.0
        t0 = time.time()
        if self.persistent_projector is not None:
            out = self._run_forward(self.persistent_projector, volume)
            self.last_projection_time = time.time() - t0
            return out
        src, dst, M, b = self._geometry(volume.device)
        Mi = self.core_module.M_inv.to(volume.device)
        pieces = []
        for s, e, table in self._ranges(volume.device):
            t1 = time.time()
            # differentiable, as the reference's per-subset module forward
            pieces.append(CTProjector3DFunction.apply(volume, *_parts(table), M, b, src[s:e], dst[s:e], self.backend,
                                                      None, Mi, None))
            self.last_projection_time += time.time() - t1
        return torch.cat(pieces, dim=-1)

    def forward_project(self, volume):
        return self.forward(volume)

    def back_project(self, sinogram):
        self.last_precompute_time = self.last_projection_time = 0.0
        t0 = time.time()
        if self.persistent_projector is not None:
            out = self._run_backward(self.persistent_projector, sinogram)
            self.last_projection_time = time.time() - t0
            return out
        src, dst, M, b = self._geometry(sinogram.device)
        Mi = self.core_module.M_inv.to(sinogram.device)
        vol = None
        for s, e, table in self._ranges(sinogram.device):
            t1 = time.time()
            part = back_project_3d_cuda(sinogram[..., s:e].contiguous(), table, src[s:e], dst[s:e], M, b, self.n_x,
                                        self.n_y, self.n_z, M_inv=Mi)
            vol = part if vol is None else vol.add_(part)
            self.last_projection_time += time.time() - t1
        return vol


class RandomSubsetProjector(SubsetProjector):
    """A random subset of the core rays (reference :231-276).  The draw is the
    reference's: ``torch.manual_seed(seed)`` (when a seed is set) and then
    ``torch.randperm(n_rays)[:subset_size]`` on the host.  The subset's rays
    are gathered into device buffers kept across draws and projected on the
    fly; with ``precomputed_intersections=True`` a module with the subset's
    tables is built instead."""

    def __init__(self, base_projector, subset_size=10000, precomputed_intersections=False, randomize_on_forward=False,
                 randomize_on_backward=False, seed=None, verbose=False):
        super().__init__(base_projector, subset_size, precomputed_intersections, verbose)
        self.randomize_on_forward = randomize_on_forward
        self.randomize_on_backward = randomize_on_backward
        self.seed = seed
        self.current_indices = None
        self._table_module = None
        self._src = self._dst = None
        self._flat = N.flat_opts()  # a random subset has no detector layout
        self.randomize_projector()

    def randomize_projector(self, subset_size=None, seed=None):
        if subset_size is not None:
            self.subset_size = subset_size
        if seed is not None:
            self.seed = seed
        if self.seed is not None:
            torch.manual_seed(self.seed)
        self.current_indices = torch.randperm(self.n_total_rays_core, device="cpu")[:self.subset_size]
        if self.precomputed_intersections:
            self._table_module = self._get_subset_module(self.current_indices)
            return
        core = self.core_module
        pick = self.current_indices.to(core.src.device)
        n = pick.numel()
        if self._src is None or self._src.shape[0] != n:
            self._src = torch.empty((n, 3), dtype=torch.float32, device=self.device)
            self._dst = torch.empty((n, 3), dtype=torch.float32, device=self.device)
        self._src.copy_(core.src.index_select(0, pick))
        self._dst.copy_(core.dst.index_select(0, pick))

    @property
    def current_subset_module(self):
        """The subset as a CTProjector3DModule (built on request when the
        subset projects on the fly)."""
        if self._table_module is not None:
            return self._table_module
        return self._get_subset_module(self.current_indices)

    def forward(self, volume):
        if self.randomize_on_forward:
            self.randomize_projector()
        if self._table_module is not None:
            return self._run_forward(self._table_module, volume)
        core = self.core_module
        return CTProjector3DFunction.apply(volume, None, None, None, core.M, core.b, self._src, self._dst,
                                           self.backend, self._flat, core.M_inv.to(volume.device), None)

    def back_project(self, sinogram):
        if self.randomize_on_backward:
            self.randomize_projector()
        if self._table_module is not None:
            return self._run_backward(self._table_module, sinogram)
        core = self.core_module
        return back_project_3d_cuda(sinogram.contiguous(), None, self._src, self._dst, core.M, core.b, self.n_x,
                                    self.n_y, self.n_z, tiling=self._flat, M_inv=core.M_inv.to(sinogram.device))

    def forward_project(self, volume):
        return self.forward(volume)
