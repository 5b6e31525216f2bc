"""CTProjector3DModule: the reference's 3-D projector nn.Module, B200 backed.

Constructor, attributes and methods follow the reference
(tomography/ct_projector_3d_module.py:28-253): ``forward`` /
``forward_project`` are differentiable (A with A^T backward),
``back_project`` is the raw adjoint (no autograd, as the preconditioners
expect), ``save_tvals`` / ``load_tvals`` read and write the same dict
``{tvals_uint16, tvals_start, tvals_scale, tvals_full, n_x, n_y, n_z, n_ray}``,
``tvals`` decompresses, ``set_tvals`` installs a table.

Differences, none in results:
 * ``precomputed_intersections=True`` builds the table on the GPU (one
   launch: per-ray stable merge of the plane runs) instead of on the CPU with
   torch.sort; the table values are identical for the diagonal affines the
   geometry classes build, and it is then trimmed and compressed with the
   reference module's encoder (compress_tvals_to_uint16 semantics).
 * M^-1 is computed once on the device and cached until M changes.
 * an optional ``ray_tiling`` launch hint (set by the cone-beam class).
 * ``deterministic_adjoint`` makes ``back_project`` and the autograd backward
   of the on-the-fly projector bitwise reproducible.  ``True`` or ``"fixed"``:
   the forward's own walk (either voxel rule, any ray layout) scattering in
   64-bit fixed point (back_project_3d_fixed_cuda).  ``"gather"`` (with a
   flat-panel table ``panels``, which the cone-beam and StaticCT classes
   build): per-voxel gathering, the exact transpose of the forward with the
   crossing voxel rule.
"""
from __future__ import annotations

import math

import torch

from .. import _C
from .. import _native as N
from ._common import InverseCache, require_cuda, voxel_diag_len
from .ct_projector_3d_autograd import CTProjector3DFunction
from .ct_projector_3d_cuda import back_project_3d_cuda, compute_intersections_3d_cuda
from .ct_projector_3d_torch import compress_tvals_to_uint16, decompress_tvals_from_uint16
from .fixed_adjoint import back_project_3d_fixed_cuda
from .gather import back_project_3d_gather_cuda

__all__ = ["CTProjector3DModule", "precompute_tvals_stitched", "adjoint_mode"]


def adjoint_mode(deterministic_adjoint) -> str:
    """'atomic', 'fixed' or 'gather' for a deterministic_adjoint argument."""
    if deterministic_adjoint in (False, None, "atomic"):
        return "atomic"
    if deterministic_adjoint is True or deterministic_adjoint == "fixed":
        return "fixed"
    if deterministic_adjoint == "gather":
        return "gather"
    raise ValueError(f"deterministic_adjoint must be False, True, 'fixed' or 'gather', got {deterministic_adjoint!r}")


def _trim_inf_columns(t: torch.Tensor) -> torch.Tensor:
    """Drop trailing columns that are +inf for every ray
    (reference ct_projector_3d_module.py:92-97)."""
    finite_cols = torch.isfinite(t).any(dim=0)
    if bool(finite_cols.all()):
        return t.contiguous()
    nz = torch.nonzero(~finite_cols)
    first = int(nz[0]) if nz.numel() else t.shape[1]
    return t[:, :first].contiguous()


class CTProjector3DModule(torch.nn.Module):
    def __init__(self, n_x, n_y, n_z, M, b, src, dst, backend="cuda", device=None, precomputed_intersections=False,
                 tvals=None, use_compression=True, ray_tiling=None, panels=None, deterministic_adjoint=False):
        super().__init__()
        if device is None:
            device = torch.device("cuda" if torch.cuda.is_available() else "cpu")
        self.backend = backend
        self.n_x, self.n_y, self.n_z = int(n_x), int(n_y), int(n_z)
        self.use_compression = use_compression
        self.ray_tiling = ray_tiling
        self._active = {}  # launch tiling -> (geometry, versions, ActiveRayOpts)
        self._minv = InverseCache()
        # the kernels read raw pointers: keep contiguous float32 copies
        f32 = lambda t: t.to(torch.float32).contiguous()  # noqa: E731
        self.register_buffer("M", f32(M))
        self.register_buffer("b", f32(b))
        self.register_buffer("src", f32(src))
        self.register_buffer("dst", f32(dst))
        self.panels = panels
        self.adjoint_mode = adjoint_mode(deterministic_adjoint)
        self.deterministic_adjoint = self.adjoint_mode != "atomic"
        if self.adjoint_mode == "gather" and panels is None:
            raise ValueError("deterministic_adjoint='gather' needs a flat-panel table (panels_from_grid)")
        self.tvals_uint16 = None
        self.tvals_start = None
        self.tvals_scale = None
        self.tvals_full = None
        self.precomputed_intersections = False
        if device is not None:
            self.to(device)
        if tvals is not None:
            self.set_tvals(tvals)
        elif precomputed_intersections:
            require_cuda(self.src, self.dst, self.M, self.b, what="geometry for precomputed intersections")
            full = compute_intersections_3d_cuda(self.n_x, self.n_y, self.n_z, self.M, self.b, self.src, self.dst,
                                                 M_inv=self.M_inv)
            full = _trim_inf_columns(full)
            if use_compression:
                self.tvals_uint16, self.tvals_start, self.tvals_scale = compress_tvals_to_uint16(
                    full, self.M, self.src, self.dst)
                del full
            else:
                self.tvals_full = full
            self.precomputed_intersections = True

    def __getstate__(self):
        # the active-tile lists are device state rebuilt on first use: not copied or pickled
        state = dict(self.__dict__)
        state["_active"] = {}
        return state

    # -- geometry helpers -------------------------------------------------
    @property
    def M_inv(self) -> torch.Tensor:
        return self._minv.get(self.M)

    def to(self, *args, **kwargs):
        super().to(*args, **kwargs)
        device = torch._C._nn._parse_to(*args, **kwargs)[0]
        if device is not None:
            for name in ("tvals_uint16", "tvals_start", "tvals_scale", "tvals_full", "panels"):
                t = getattr(self, name, None)
                if isinstance(t, torch.Tensor):
                    setattr(self, name, t.to(device))
        return self

    def _launch_tiling(self):
        """ray_tiling with the list of its active tiles (active_tiling_for)."""
        if self._table()[0] is not None:
            return self.ray_tiling
        return self.active_tiling_for(self.ray_tiling)

    def active_tiling_for(self, t):
        """Launch tiling `t` of this scan with the list of its active tiles
        (the tiles holding a ray that the walks charge,
        _native.active_tiling), computed once per geometry and tiling: the
        on-the-fly launches then skip the tiles whose rays all miss the
        volume, with the same results.  `t` itself for a flat launch."""
        if t is None or t.n_view == 0 or not self.src.is_cuda:
            return t
        geom = (self.src, self.dst, self.M, self.b)
        tkey = tuple(getattr(t, f) for f, _ in N.RayOpts._fields_)
        versions = (tuple(g._version for g in geom), self.n_x, self.n_y, self.n_z)
        hit = self._active.get(tkey)
        if hit is not None and hit[1] == versions and all(a is b for a, b in zip(hit[0], geom)):
            return hit[2]
        opts = N.active_tiling(t, self.src, self.dst, self.M_inv, self.b, (self.n_x, self.n_y, self.n_z))
        if len(self._active) >= 8:  # a few launch shapes at most
            self._active.clear()
        self._active[tkey] = (geom, versions, opts)
        return opts

    def _panels(self):
        return self.panels if (self.adjoint_mode == "gather" and self._table()[0] is None) else None

    def _fixed(self) -> bool:
        return self.adjoint_mode == "fixed" and self._table()[0] is None

    def _table(self):
        if self.tvals_uint16 is not None:
            return self.tvals_uint16, self.tvals_start, self.tvals_scale
        return self.tvals_full, None, None

    def _ensure_table_device(self, device):
        for name in ("tvals_uint16", "tvals_start", "tvals_scale", "tvals_full"):
            t = getattr(self, name)
            if isinstance(t, torch.Tensor) and t.device != device:
                setattr(self, name, t.to(device))

    # -- projector ------------------------------------------------------
    def forward(self, volume):
        require_cuda(volume, what="volume")
        self._ensure_table_device(volume.device)
        t_main, t_start, t_scale = self._table()
        return CTProjector3DFunction.apply(volume, t_main, t_start, t_scale, self.M, self.b, self.src, self.dst,
                                           self.backend, self._launch_tiling(), self.M_inv, self._panels(),
                                           self._fixed())

    def forward_project(self, volume):
        return self.forward(volume)

    def back_project(self, sinogram):
        require_cuda(sinogram, what="sinogram")
        self._ensure_table_device(sinogram.device)
        t_main, t_start, t_scale = self._table()
        tv = (t_main, t_start, t_scale) if t_start is not None else t_main
        with torch.no_grad():
            if self._panels() is not None:
                return back_project_3d_gather_cuda(sinogram, self.src, self.dst, self.M, self.b, self.n_x, self.n_y,
                                                   self.n_z, self.panels, M_inv=self.M_inv)
            if self._fixed():
                return back_project_3d_fixed_cuda(sinogram.contiguous(), self.src, self.dst, self.M, self.b, self.n_x,
                                                  self.n_y, self.n_z, tiling=self._launch_tiling(), M_inv=self.M_inv)
            return back_project_3d_cuda(sinogram.contiguous(), tv, self.src, self.dst, self.M, self.b, self.n_x,
                                        self.n_y, self.n_z, tiling=self._launch_tiling(), M_inv=self.M_inv)

    # -- tvals lifecycle (reference :190-253) ------------------------------
    def save_tvals(self, filePath):
        if self.tvals_uint16 is None and self.tvals_full is None:
            raise ValueError("No precomputed t-values to save.")
        cpu = lambda t: t.cpu() if t is not None else None  # noqa: E731
        torch.save({
            "tvals_uint16": cpu(self.tvals_uint16), "tvals_start": cpu(self.tvals_start),
            "tvals_scale": cpu(self.tvals_scale), "tvals_full": cpu(self.tvals_full),
            "n_x": self.n_x, "n_y": self.n_y, "n_z": self.n_z, "n_ray": self.src.shape[0],
        }, filePath)

    def load_tvals(self, filePath, device=None):
        if device is None:
            device = self.src.device
        d = torch.load(filePath, map_location="cpu")
        if d["n_x"] != self.n_x or d["n_y"] != self.n_y or d["n_z"] != self.n_z:
            raise ValueError("Dimension mismatch")
        for name in ("tvals_uint16", "tvals_start", "tvals_scale", "tvals_full"):
            t = d.get(name)
            setattr(self, name, t.to(device) if t is not None else None)
        self.precomputed_intersections = True

    def set_tvals(self, tvals, device=None):
        if device is None:
            device = self.src.device
        if tvals is None:
            self.tvals_uint16 = self.tvals_start = self.tvals_scale = self.tvals_full = None
            self.precomputed_intersections = False
            return
        if isinstance(tvals, (tuple, list)):
            tu16, tstart, tscale = tvals
            self.tvals_uint16, self.tvals_start, self.tvals_scale = tu16.to(device), tstart.to(device), \
                tscale.to(device)
            self.tvals_full = None
        elif self.use_compression:
            t = tvals.to(device)
            self.tvals_uint16, self.tvals_start, self.tvals_scale = compress_tvals_to_uint16(t, self.M, self.src,
                                                                                             self.dst)
            self.tvals_full = None
        else:
            self.tvals_full = tvals.to(device)
            self.tvals_uint16 = self.tvals_start = self.tvals_scale = None
        self.precomputed_intersections = True

    @property
    def tvals(self):
        if self.tvals_uint16 is not None:
            return decompress_tvals_from_uint16(self.tvals_uint16, self.tvals_start, self.tvals_scale)
        return self.tvals_full

    @tvals.setter
    def tvals(self, value):
        self.set_tvals(value)


def precompute_tvals_stitched(n_x, n_y, n_z, M, b, src_all, dst_all, chunk_size=1000000, backend="cuda",
                              device=None, verbose=True, use_compression=True):
    """Tables for all rays in chunks, returned on the CPU like the reference
    (ct_projector_3d_module.py:256-315): int16 [n_ray, n_int] + starts +
    scales, or a float [n_ray, n_int] table, n_int = (n_x+1)+(n_y+1)+(n_z+1).
    Chunks are built on the GPU; ``backend='cuda'`` encodes with the reference
    CUDA encoder (as the reference's cuda path does), ``backend='torch'`` with
    its torch encoder."""
    if device is None:
        device = torch.device("cuda")
    device = torch.device(device)
    if device.type != "cuda":
        raise RuntimeError("ct_laboratory_b200: precompute runs on a CUDA device")
    n_ray = src_all.shape[0]
    n_int = (n_x + 1) + (n_y + 1) + (n_z + 1)
    if verbose:
        print(f"Precomputing {n_ray} rays in chunks of {chunk_size} using {backend}...")
    M_d, b_d = M.to(device), b.to(device)
    Mi = InverseCache().get(M_d if M_d.dim() == 2 else M_d[0])
    vdl = voxel_diag_len(M_d) if use_compression else None
    if use_compression:
        main = torch.zeros((n_ray, n_int), dtype=torch.int16)
        starts = torch.zeros(n_ray, dtype=torch.float32)
        scales = torch.zeros(n_ray, dtype=torch.float32)
    else:
        full = torch.zeros((n_ray, n_int), dtype=torch.float32)
    for i in range(math.ceil(n_ray / chunk_size)):
        s, e = i * chunk_size, min((i + 1) * chunk_size, n_ray)
        src_c = src_all[s:e].to(device).float().contiguous()
        dst_c = dst_all[s:e].to(device).float().contiguous()
        t_c = _C.compute_intersections_3d(n_x, n_y, n_z, src_c, dst_c, Mi,
                                          (b_d if b_d.dim() == 1 else b_d[0]).float().contiguous())
        if use_compression:
            mode = 0 if backend == "cuda" else 1
            if mode == 1:
                diag_t = voxel_diag_len(M.cpu() if M.dim() == 2 else M[0].cpu())
            else:
                diag_t = vdl
            t16, ts, tsc = _C.compress_tvals_3d_mode(t_c, src_c, dst_c, diag_t, mode=mode)
            main[s:e] = t16.cpu()
            starts[s:e] = ts.cpu()
            scales[s:e] = tsc.cpu()
        else:
            full[s:e] = t_c.cpu()
        del src_c, dst_c, t_c
    if use_compression:
        return main.contiguous(), starts, scales
    return full.contiguous()
