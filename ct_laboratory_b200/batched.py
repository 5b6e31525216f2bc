"""Many scans projected in one persistent launch, with an autotuner and
CUDA-graph replay.

``ScanBatch(projectors)`` binds a list of 2-D projectors
(``CTProjector2DModule`` and its fan-beam / StaticCT subclasses) or of 3-D
projectors (``CTProjector3DModule`` and subclasses) to device buffers it
allocates once:

  images_in[i]   forward input of scan i          ([n_row, n_col] or [n_x, n_y, n_z])
  sinos_out[i]   forward output                   ([n_ray])
  sinos_in[i]    adjoint input                    ([n_ray])
  images_out[i]  adjoint output                   (same shape as images_in[i])

(or binds caller-owned tensors given as ``buffers={"images_in": [...], ...}``).

``forward()`` computes every sinos_out[i] = A_i images_in[i] in one launch
of persistent CTAs whose warps pull slices of the ray tiles of all scans
from a device work counter (libctlab_b200.so
``ctlab_forward_project_batched``); ``back()`` the adjoints likewise, each
direction with its own plan and tile layout.  ``forward_loop()`` / ``back_loop()`` run the very same
walks one scan at a time through the single-scan entry points, into the
same buffers: the per-instance loop the batch replaces.  Forward results are
bitwise equal between the two; adjoints up to the order of float atomics,
or bitwise with ``deterministic_adjoint=True`` (3-D: each scan's adjoint
scatters in 64-bit fixed point, scan by scan).

Each direction has a mode: the persistent launch, or the loop of
single-scan launches (the default for the 3-D forward, where the
single-scan column walk is faster on large scans).  Tile shapes (rays per
CTA and how they are laid over each scan's detector) and the modes are
chosen by ``autotune()``, which times the candidates on the batch itself
and caches the winner per batch signature.  ``capture()`` records forward
and / or adjoint into a ``torch.cuda.CUDAGraph`` for replay.

The reference has no batched launch: its projector modules take one scan
per call (tomography/ct_projector_3d_module.py:171-188,
ct_projector_2d_module.py:50-65).
"""
from __future__ import annotations

import ctypes
import statistics

import torch

from . import _native as N
from .tomography.ct_projector_3d_module import CTProjector3DModule

__all__ = ["ScanBatch", "Autotuner", "tile_kinds"]


def _ndim(p):
    return 3 if isinstance(p, CTProjector3DModule) else 2


def _dims(p):
    return (p.n_x, p.n_y, p.n_z) if _ndim(p) == 3 else (p.n_row, p.n_col)


def _ray_grid(p):
    """(n_view, n_bin) when the projector's rays are ordered [view][bin] with
    n_bin detector cells per view, else None."""
    n_ray = int(p.src.shape[0])
    if hasattr(p, "n_view") and hasattr(p, "n_det"):  # fan-beam: [view][cell]
        bins = int(p.n_det)
    elif hasattr(p, "n_module") and hasattr(p, "det_n_col"):  # uniform StaticCT ring: [source][module][col]
        bins = int(p.n_module) * int(p.det_n_col)
    else:
        return None
    if bins <= 0 or n_ray % bins:
        return None
    return n_ray // bins, bins


def tile_kinds(p):
    """Tile layouts that apply to projector p (the autotuner's choices).

    flat      consecutive rays, block_threads per CTA
    grid32    2-D: 32 detector cells x (block_threads/32) views per CTA, lanes
              along cells (neighbouring rays: coherent gathers, the forward's
              choice)
    grid64    2-D: 64 cells x (block_threads/64) views
    vgrid32   2-D: 32 views x (block_threads/32) cells, lanes along views (the
              same cell seen from 32 directions: the lanes' pixels are far
              apart)
    vgrid64   2-D: 64 views x (block_threads/64) cells
    col32     3-D detector grid: 32 detector rows x (block_threads/32) columns
              (lanes of a warp down one detector column: the column walk)
    col64     3-D: 64 rows x (block_threads/64) columns
    col16     3-D detector grid of 16 rows per column (StaticCT modules):
              16 rows x (block_threads/16) columns, the column walk in two
              16-lane groups per warp
    """
    kinds = ["flat"]
    if _ndim(p) == 2:
        if _ray_grid(p) is not None:
            kinds += ["grid32", "grid64", "vgrid32", "vgrid64"]
    elif getattr(p, "ray_tiling", None) is not None and p.ray_tiling.n_view > 0:
        kinds += ["col16"] if p.ray_tiling.n_row == 16 else ["col32", "col64"]
    return kinds


def _opts(p, kind, voxel_rule, block_threads):
    """RayOpts of projector p laid out as `kind` (falls back to flat when the
    kind does not apply or does not fit block_threads)."""
    rows = {"grid32": 32, "grid64": 64, "vgrid32": 32, "vgrid64": 64, "col32": 32, "col64": 64,
            "col16": 16}.get(kind)
    if rows is None or rows > block_threads or kind not in tile_kinds(p):
        return N.flat_opts(voxel_rule=voxel_rule, block_threads=block_threads)
    if kind.startswith("grid"):
        n_view, n_bin = _ray_grid(p)
        # rows = detector cells (stride 1), columns = views (stride n_bin)
        return N.tiling(1, n_bin, n_view, n_bin * n_view, 1, n_bin, tile_rows=rows, block_threads=block_threads,
                        voxel_rule=voxel_rule)
    if kind.startswith("vgrid"):
        n_view, n_bin = _ray_grid(p)
        # rows = views (stride n_bin), columns = detector cells (stride 1)
        return N.tiling(1, n_view, n_bin, n_bin * n_view, n_bin, 1, tile_rows=rows, block_threads=block_threads,
                        voxel_rule=voxel_rule)
    t = p.ray_tiling
    return N.tiling(t.n_view, t.n_row, t.n_col, t.view_stride, t.row_stride, t.col_stride, tile_rows=rows,
                    block_threads=block_threads, voxel_rule=voxel_rule)


def _cost(p):
    """Rough cost of one ray of p (planes it may cross): heavy scans go first."""
    return sum(_dims(p))


class ScanBatch:
    def __init__(self, projectors, voxel_rule=N.VOXEL_CROSSING, forward=True, adjoint=True, block_threads=256,
                 kind="auto", buffers=None, deterministic_adjoint=False, fixed_workspace=None):
        self.projectors = list(projectors)
        if not self.projectors:
            raise ValueError("ScanBatch needs at least one projector")
        nd = {_ndim(p) for p in self.projectors}
        if len(nd) != 1:
            raise ValueError("ScanBatch: all projectors must be 2-D or all 3-D")
        self.ndim = nd.pop()
        self.device = self.projectors[0].src.device
        if self.device.type != "cuda":
            raise RuntimeError("ScanBatch: projectors must live on a CUDA device (there is no CPU implementation)")
        self.voxel_rule = int(voxel_rule)
        self.has_forward, self.has_adjoint = bool(forward), bool(adjoint)
        # reproducible adjoint (3-D): every scan's walk scatters in 64-bit fixed
        # point (ctlab_back_project_3d_fixed) into one int64 workspace reused
        # scan after scan, so a scan's volume is the same bits whichever other
        # scans share the batch
        self.deterministic_adjoint = bool(deterministic_adjoint)
        self._fixed_ws = None
        if self.deterministic_adjoint and adjoint:
            if self.ndim != 3:
                raise ValueError("ScanBatch: deterministic_adjoint is implemented for 3-D scans")
            need = max(int(N.lib.ctlab_back_project_3d_fixed_workspace_bytes(1, *_dims(p))) for p in self.projectors)
            if fixed_workspace is not None:  # a caller-owned buffer, reused from batch to batch
                if (fixed_workspace.dtype != torch.uint8 or fixed_workspace.device != self.device
                        or fixed_workspace.numel() < need):
                    raise ValueError(f"ScanBatch: fixed_workspace must be a uint8 tensor of >= {need} bytes on "
                                     f"{self.device}")
                self._fixed_ws = fixed_workspace
            else:
                self._fixed_ws = torch.empty(need, dtype=torch.uint8, device=self.device)
        shapes = [_dims(p) for p in self.projectors]
        n_rays = [int(p.src.shape[0]) for p in self.projectors]
        if buffers is None:
            self.images_in = self._arena(shapes) if forward else None
            self.sinos_out = self._arena([(n,) for n in n_rays]) if forward else None
            self.sinos_in = self._arena([(n,) for n in n_rays]) if adjoint else None
            self.images_out = self._arena(shapes) if adjoint else None
        else:
            # caller-owned tensors (e.g. the state of reconstruction jobs): one
            # per scan, float32, contiguous, on the projectors' device
            want = {"images_in": (forward, shapes), "sinos_out": (forward, [(n,) for n in n_rays]),
                    "sinos_in": (adjoint, [(n,) for n in n_rays]), "images_out": (adjoint, shapes)}
            for name, (used, shp) in want.items():
                ts = buffers.get(name) if used else None
                if used:
                    if ts is None or len(ts) != len(shp):
                        raise ValueError(f"ScanBatch: buffers['{name}'] needs one tensor per scan")
                    for tt, s in zip(ts, shp):
                        if (tt.dtype != torch.float32 or not tt.is_contiguous() or tt.device != self.device
                                or tt.numel() != int(torch.Size(s).numel())):
                            raise ValueError(f"ScanBatch: buffers['{name}'] must be contiguous float32 tensors of "
                                             f"shape {tuple(s)} on {self.device}")
                setattr(self, name, list(ts) if used else None)
        # 2-D adjoint: a transposed scratch image per scan
        self.scratch = self._arena(shapes) if adjoint and self.ndim == 2 else None
        # heaviest rays first: long tiles start early, short ones fill the tail
        self.order = sorted(range(len(self.projectors)), key=lambda i: -_cost(self.projectors[i]))
        nbytes = N.lib.ctlab_batch_workspace_bytes(len(self.projectors))
        if nbytes < 0:
            raise ValueError(f"ScanBatch: {len(self.projectors)} scans is outside [1, 65535]")
        # one plan (and workspace) per direction: the forward and the adjoint
        # may lay their tiles out differently
        self._ws_bytes = int(nbytes)
        self._ws, self._ws_ptr, self._plans = {}, {}, {}
        for d in ("fwd", "adj"):
            self._ws[d] = torch.empty(self._ws_bytes + 256, dtype=torch.uint8, device=self.device)
            self._ws_ptr[d] = self._ws[d].data_ptr() + (-self._ws[d].data_ptr()) % 256
            self._plans[d] = N.Batch()
        self.config = None
        self.config_adj = None
        self.configure(block_threads=block_threads, kind=kind)

    # ------------------------------------------------------------ buffers
    def _arena(self, shapes):
        """One allocation holding a zeroed tensor per shape, each 256-byte aligned."""
        sizes = [int(torch.Size(s).numel()) for s in shapes]
        pad = lambda n: (n + 63) // 64 * 64  # noqa: E731  (64 floats = 256 bytes)
        total = sum(pad(n) for n in sizes)
        flat = torch.zeros(max(total, 1), dtype=torch.float32, device=self.device)
        out, off = [], 0
        for s, n in zip(shapes, sizes):
            out.append(flat[off:off + n].view(s))
            off += pad(n)
        return out

    # ------------------------------------------------------------ planning
    def _scan(self, i, kind, block_threads):
        p = self.projectors[i]
        s = N.Scan()
        if self.has_forward:
            s.image_in, s.sino_out = self.images_in[i].data_ptr(), self.sinos_out[i].data_ptr()
        if self.has_adjoint:
            s.sino_in, s.image_out = self.sinos_in[i].data_ptr(), self.images_out[i].data_ptr()
            if self.scratch is not None:
                s.image_scratch = self.scratch[i].data_ptr()
        s.src, s.dst = p.src.data_ptr(), p.dst.data_ptr()
        s.M_inv, s.b = p.M_inv.data_ptr(), p.b.data_ptr()
        s.n_ray = int(p.src.shape[0])
        d = _dims(p)
        for a in range(3):
            s.dims[a] = int(d[a]) if a < len(d) else 0
        s.ndim = self.ndim
        k = kind if isinstance(kind, str) else kind[i]
        s.opts = _opts(p, k, self.voxel_rule, block_threads)
        return s

    def _default_kinds(self, direction):
        out = []
        for p in self.projectors:
            k = tile_kinds(p)
            if "col16" in k:
                out.append("col16")
            elif "col32" in k:
                out.append("col32")
            elif "grid32" in k:
                out.append("grid32")
            else:
                out.append("flat")
        return out

    def configure(self, block_threads=256, kind="auto", n_cta=0, direction="both", mode="auto"):
        """(Re)plan the batch with a tile layout: `kind` is one tile kind for
        every scan or a list with one kind per scan; "auto" takes col32 for
        detector grids in 3-D (col16 for 16 rows per column), grid32 for 2-D view x cell grids (neighbouring
        rays in a warp: coherent gathers, and adjoint reductions into
        neighbouring pixels of one row), else flat.  `direction` ("fwd", "adj" or "both")
        selects the plan(s) to replace.  `mode` is how forward() / back() run
        that direction: "persistent" (one launch over all scans) or "loop"
        (the single-scan kernels scan by scan, with the same tile layouts);
        "auto" takes the loop for the 3-D forward, whose single-scan column
        walk is faster than the persistent kernel's on scans of millions of
        rays (8.75 against 9.98 ms on the cone256 scan), and for the 3-D
        adjoint when every scan has at least 2^20 rays; the persistent launch
        otherwise.  3-D loop launches take each projector's active-tile
        list (CTProjector3DModule.active_tiling_for).  Returns the forward configuration (the adjoint's
        is ``config_adj``)."""
        if mode not in ("auto", "persistent", "loop"):
            raise ValueError(f"ScanBatch: mode must be 'auto', 'persistent' or 'loop' (got {mode!r})")
        for d in (("fwd", "adj") if direction == "both" else (direction,)):
            k = self._default_kinds(d) if kind == "auto" else kind
            arr = (N.Scan * len(self.projectors))(*[self._scan(i, k, block_threads) for i in self.order])
            with torch.cuda.device(self.device):
                N.call("ctlab_batch_plan", arr, len(self.projectors), int(block_threads),
                       ctypes.c_void_p(self._ws_ptr[d]), self._ws_bytes, ctypes.byref(self._plans[d]),
                       N.stream_of(self._ws[d]))
                ctas = n_cta
                if ctas == 0:
                    v = ctypes.c_int32(0)
                    N.call("ctlab_batch_default_ctas", self.ndim, int(d == "adj"), self.voxel_rule,
                           int(block_threads), ctypes.byref(v))
                    ctas = v.value
            # auto: 3-D scans run one launch each (with their active-tile
            # lists) where every scan fills the GPU on its own (>= 2^20 rays:
            # the adjoint of four serving-size scans, 23.6 against 26.1 ms
            # persistent); the persistent launch otherwise, for batches of
            # small scans
            big = all(int(p.src.shape[0]) >= (1 << 20) for p in self.projectors)
            m = mode if mode != "auto" else (
                "loop" if self.ndim == 3 and (d == "fwd" or big) else "persistent")
            if d == "adj" and self._fixed_ws is not None:
                m = "loop"  # the fixed-point adjoint runs scan by scan
            cfg = {"block_threads": int(block_threads), "kind": k, "n_cta": int(ctas), "mode": m}
            opts = [_opts(self.projectors[i], k if isinstance(k, str) else k[i], self.voxel_rule, block_threads)
                    for i in range(len(self.projectors))]
            if self.ndim == 3 and m == "loop":
                # the per-scan launches skip each scan's tiles whose rays all
                # miss its volume (lists cached on the projector)
                opts = [self.projectors[i].active_tiling_for(o) for i, o in enumerate(opts)]
            if d == "fwd":
                self.config, self._loop_opts_f = cfg, opts
            else:
                self.config_adj, self._loop_opts_a = cfg, opts
        return self.config

    @property
    def total_tiles(self):
        return int(self._plans["fwd"].total_tiles)

    # ------------------------------------------------------------ launches
    def forward(self):
        """sinos_out[i] = A_i images_in[i] for every scan: one launch, or the
        per-scan loop when the forward's mode is "loop"."""
        if self.config["mode"] == "loop":
            return self.forward_loop()
        with torch.cuda.device(self.device):
            N.call("ctlab_forward_project_batched", ctypes.byref(self._plans["fwd"]), self.config["n_cta"],
                   N.stream_of(self._ws["fwd"]))

    def back(self, accumulate=False):
        """images_out[i] (+)= A_i^T sinos_in[i] for every scan: one zeroing
        launch (unless accumulating) and one persistent launch (and for 2-D
        scans the add-back of the transposed scratch), or the per-scan loop
        when the adjoint's mode is "loop"."""
        if self.config_adj["mode"] == "loop":
            return self.back_loop(accumulate)
        with torch.cuda.device(self.device):
            N.call("ctlab_back_project_batched", ctypes.byref(self._plans["adj"]), int(bool(accumulate)),
                   self.config_adj["n_cta"], N.stream_of(self._ws["adj"]))

    def forward_loop(self):
        """The same forward one scan at a time (single-scan entry points)."""
        st = N.stream_of(self._ws["fwd"])
        with torch.cuda.device(self.device):
            for i, p in enumerate(self.projectors):
                o = self._loop_opts_f[i]
                act = getattr(o, "active", None)
                if self.ndim == 3 and act is not None:
                    N.call("ctlab_forward_project_3d_on_the_fly_tiles", N.ptr(self.images_in[i]), 1, p.n_x, p.n_y,
                           p.n_z, N.ptr(p.src), N.ptr(p.dst), int(p.src.shape[0]), N.ptr(p.M_inv), N.ptr(p.b),
                           N.ptr(self.sinos_out[i]), ctypes.byref(o), N.ptr(act[0]), act[1], st)
                elif self.ndim == 3:
                    N.call("ctlab_forward_project_3d_on_the_fly_ex", N.ptr(self.images_in[i]), 1, p.n_x, p.n_y,
                           p.n_z, N.ptr(p.src), N.ptr(p.dst), int(p.src.shape[0]), N.ptr(p.M_inv), N.ptr(p.b),
                           N.ptr(self.sinos_out[i]), ctypes.byref(o), st)
                else:
                    N.call("ctlab_forward_project_2d_siddon", N.ptr(self.images_in[i]), 1, p.n_row, p.n_col,
                           N.ptr(p.src), N.ptr(p.dst), int(p.src.shape[0]), N.ptr(p.M_inv), N.ptr(p.b),
                           N.ptr(self.sinos_out[i]), ctypes.byref(o), st)

    def back_loop(self, accumulate=False):
        """The same adjoint one scan at a time (single-scan entry points)."""
        st = N.stream_of(self._ws["adj"])
        acc = int(bool(accumulate))
        with torch.cuda.device(self.device):
            for i, p in enumerate(self.projectors):
                o = self._loop_opts_a[i]
                act = getattr(o, "active", None)
                tiles, n_tiles = (N.ptr(act[0]), act[1]) if act is not None else (None, -1)
                if self._fixed_ws is not None:
                    N.call("ctlab_back_project_3d_fixed", N.ptr(self.sinos_in[i]), 1, int(p.src.shape[0]),
                           N.ptr(p.src), N.ptr(p.dst), N.ptr(p.M_inv), N.ptr(p.b), p.n_x, p.n_y, p.n_z,
                           N.ptr(self.images_out[i]), acc, ctypes.byref(o), tiles, n_tiles, N.ptr(self._fixed_ws),
                           self._fixed_ws.numel(), st)
                elif self.ndim == 3 and act is not None:
                    N.call("ctlab_back_project_3d_on_the_fly_tiles", N.ptr(self.sinos_in[i]), 1, int(p.src.shape[0]),
                           N.ptr(p.src), N.ptr(p.dst), N.ptr(p.M_inv), N.ptr(p.b), p.n_x, p.n_y, p.n_z,
                           N.ptr(self.images_out[i]), acc, ctypes.byref(o), tiles, n_tiles, st)
                elif self.ndim == 3:
                    N.call("ctlab_back_project_3d_on_the_fly_ex", N.ptr(self.sinos_in[i]), 1, int(p.src.shape[0]),
                           N.ptr(p.src), N.ptr(p.dst), N.ptr(p.M_inv), N.ptr(p.b), p.n_x, p.n_y, p.n_z,
                           N.ptr(self.images_out[i]), acc, ctypes.byref(o), st)
                else:
                    scratch = self.scratch[i] if self.scratch is not None else None
                    N.call("ctlab_back_project_2d_siddon_ws", N.ptr(self.sinos_in[i]), 1, int(p.src.shape[0]),
                           N.ptr(p.src), N.ptr(p.dst), N.ptr(p.M_inv), N.ptr(p.b), p.n_row, p.n_col,
                           N.ptr(self.images_out[i]), acc, ctypes.byref(o), N.ptr(scratch), st)

    def capture(self, forward=True, adjoint=True, accumulate=False):
        """A CUDA graph of one forward and / or adjoint pass of the batch
        (replay with .replay(); the bound buffers must stay in place)."""
        with torch.cuda.device(self.device):
            side = torch.cuda.Stream(self.device)
            side.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.stream(side):  # warm-up outside the capture
                if forward:
                    self.forward()
                if adjoint:
                    self.back(accumulate)
            torch.cuda.current_stream(self.device).wait_stream(side)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                if forward:
                    self.forward()
                if adjoint:
                    self.back(accumulate)
        return g

    def autotune(self, reps=3, block_threads=(128, 256), tuner=None):
        """Pick the fastest (block_threads, tile kind) for this batch, for the
        forward and for the adjoint separately, by timing passes; the result
        is cached per batch signature."""
        return (tuner or DEFAULT_TUNER).tune(self, reps=reps, block_threads=block_threads)

    def signature(self):
        return (self.ndim, self.voxel_rule, self.has_forward, self.has_adjoint,
                tuple((_dims(p), int(p.src.shape[0]), tuple(tile_kinds(p))) for p in self.projectors))


class Autotuner:
    """Times every candidate launch shape of a batch with CUDA events (median
    of `reps` passes after one warm-up), forward and adjoint separately, and
    keeps the fastest of each per batch signature."""

    def __init__(self):
        self.cache = {}
        self.trials = {}

    def candidates(self, batch, block_threads):
        kinds = sorted({k for p in batch.projectors for k in tile_kinds(p)})
        return [(bt, k, m) for m in ("persistent", "loop") for bt in block_threads for k in kinds]

    def _time(self, fn, device, reps):
        fn()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize(device)
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    def tune(self, batch, reps=3, block_threads=(128, 256)):
        key = batch.signature()
        if key not in self.cache:
            best, trials = {}, {}
            with torch.cuda.device(batch.device):
                for d, used, fn in (("fwd", batch.has_forward, batch.forward), ("adj", batch.has_adjoint, batch.back)):
                    if not used:
                        continue
                    res = []
                    for bt, kind, mode in self.candidates(batch, block_threads):
                        batch.configure(block_threads=bt, kind=kind, direction=d, mode=mode)
                        res.append((self._time(fn, batch.device, reps), bt, kind, mode))
                    res.sort()
                    trials[d] = res
                    best[d] = {"block_threads": res[0][1], "kind": res[0][2], "mode": res[0][3]}
            self.trials[key] = trials
            self.cache[key] = best
        for d, cfg in self.cache[key].items():
            batch.configure(block_threads=cfg["block_threads"], kind=cfg["kind"], direction=d, mode=cfg["mode"])
        return batch.config


DEFAULT_TUNER = Autotuner()
