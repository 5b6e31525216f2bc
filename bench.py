#!/usr/bin/env python
"""Benchmark of the Siddon forward projector A and its adjoint A^T on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload cone256]

A step is one forward + adjoint pair over the whole scan of the workload
(default cone256: 256^3 volume at 0.5 mm, 360 views of 512x384 cells,
70,778,880 rays; seeded synthetic ellipsoid phantom).  The metric is
GRays/s fwd+adj = rays / (t_fwd + t_adj) / 1e9.

ours (default): device-resident timing with CUDA events on the launching
stream, W untimed warm-up steps, then K timed steps; L2 is flushed (a
512 MiB write) before every timed step and the flush is not timed.  With
N > 1 (torchrun, one process per GPU) the scan's views are split across the
ranks (RaySharded3DProjector: each rank projects its whole views, the forward
all-gathers the sinogram shards and the adjoint all-reduces the partial
volumes over NCCL; strong scaling, one scan per job; --sharded takes the same
path on one GPU); --replicas instead gives every rank its own whole scan
(weak scaling, no collective).  The time is the max over ranks.  Rank 0
prints one JSON line that also holds:
  roofline      dominant kernel: algorithmic bytes / mean launch time vs the
                measured HBM copy bandwidth (MEASURED_PEAKS.json)
  cpu_baseline  the CPU port of the reference's torch path (oracle/) on this
                host's cores, on a bounded sample of views (N = 1 only)
  e2e           the same metric through the public module API with pinned
                host buffers, H2D of each step's inputs and D2H of its outputs
                inside the timed region (inputs double-buffered, uploads and
                downloads each on a stream of its own, under the kernels)
  clocks        nvidia-smi SM clock / throttle reasons sampled while timing
and, at N = 1, three legs of the other workloads (each can be switched off):
  batched       64 uneven 2-D scans: one persistent launch per direction from
                a CUDA graph against the per-scan loop (--batched-steps 0)
  serving       100 MAP jobs arriving at 20/s: the continuous-batching server
                against the plain per-job estimator loop (--serve-jobs 0)
  map           MAP on the cone scan: Lanczos k=64 preconditioner, 50
                iterations, finite-difference gradient check, adjoint
                identity (--map-iters 0)

reference: times the reference's CPU projector (the oracle's port of its
torch path) on the host cores, rank 0 only, K steps each a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Algorithmic segment counts (sum over rays of in-volume Siddon segments),
# frozen from the FP64 oracle: `python oracle/count_segments.py <workload>`.
SEGMENTS = {
    "fan256": 45_364_441,
    "cone256": 6_962_229_058,
    "batch64": 3_042_757_788,
    "static512": 1_784_871_631,
}
METRIC = "GRays/s fwd+adj"
L2_FLUSH_BYTES = 512 << 20


# --------------------------------------------------------------------------- helpers
def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback 6.65 TB/s"


def algorithmic_bytes(workload, n_ray):
    """Per launch, fwd or adj: 4 B per in-volume segment (one voxel read or
    one accumulation) + 4 B per ray (sinogram write or read)."""
    seg = SEGMENTS.get(workload)
    if seg is None:
        return None, None
    return 4 * seg + 4 * n_ray, seg


class ClockSampler:
    """nvidia-smi SM clock and throttle reasons, sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 or (args.sharded and args.impl == "ours"):
        import datetime
        import socket
        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
            # NCCL's communicator set-up lines (ranks, transports) on stderr
            os.environ.setdefault("NCCL_DEBUG", "INFO")
            os.environ.setdefault("NCCL_DEBUG_SUBSYS", "INIT")
        if world == 1:  # a one-rank group for the sharded path on one GPU
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            if "MASTER_PORT" not in os.environ:
                with socket.socket() as sk:
                    sk.bind(("127.0.0.1", 0))
                    os.environ["MASTER_PORT"] = str(sk.getsockname()[1])
            os.environ.setdefault("RANK", "0")
            os.environ.setdefault("WORLD_SIZE", "1")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    elif args.impl == "ours":
        torch.cuda.set_device(local)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# --------------------------------------------------------------------------- CPU legs
def cpu_threads():
    n = len(os.sched_getaffinity(0))
    return max(1, min(n, 64))


class CpuCase:
    """Host copies of a workload's geometry and phantom for the CPU legs."""

    def __init__(self, w, src=None, dst=None, M=None, b=None, vol=None):
        from oracle import oracle as O
        if src is None:
            src, dst, M, b = w.geometry()
        self.w = w
        self.src = np.ascontiguousarray(src.cpu().numpy() if torch.is_tensor(src) else src)
        self.dst = np.ascontiguousarray(dst.cpu().numpy() if torch.is_tensor(dst) else dst)
        self.M = np.asarray(M.cpu().numpy() if torch.is_tensor(M) else M, dtype=np.float64)
        self.Mi = O.minv(M.cpu().numpy() if torch.is_tensor(M) else M)
        self.b = np.ascontiguousarray(b.cpu().numpy() if torch.is_tensor(b) else b)
        if vol is None:
            vol = w.phantom(device="cuda" if torch.cuda.is_available() else "cpu")
        self.vol = np.ascontiguousarray(vol.cpu().numpy() if torch.is_tensor(vol) else vol)
        self.per_view = w.n_ray // w.n_view

    def rate(self, views, threads):
        """Rays/s of the oracle's port of the reference CPU path (intersections
        + sort + segment sum, then the scatter adjoint) on the given views."""
        from oracle import oracle as O
        O.set_threads(threads)
        idx = np.concatenate([np.arange(v * self.per_view, (v + 1) * self.per_view) for v in views])
        s, d = self.src[idx], self.dst[idx]
        y = np.random.default_rng(0).random(idx.size).astype(np.float32)
        t0 = time.perf_counter()
        O.fwd_otf_torch(self.vol, self.Mi, self.b, s, d)
        O.back_otf_torch(y, self.Mi, self.b, s, d, self.vol.shape)
        dt = time.perf_counter() - t0
        return idx.size / dt, idx.size, dt


def cpu_baseline(case, target_s=15.0, gpu_view0=None):
    """The oracle's port of the reference CPU path, timed; and, when the GPU
    results for view 0 are given (forward sinogram of that view, adjoint of
    that view's sinogram alone, and that sinogram), their errors against the
    FP64 oracle (the reference's plane-sort Siddon in double precision) on
    that full-size view."""
    from oracle import oracle as O
    w = case.w
    threads = cpu_threads()
    rate, n, dt = case.rate([0], threads)  # calibration: one view
    n_views = int(max(1, min(w.n_view, math.floor(target_s * rate / case.per_view))))
    views = [int(round(i * w.n_view / n_views)) % w.n_view for i in range(n_views)]
    rate, n, dt = case.rate(views, threads)
    out = {"value": rate / 1e9, "unit": "GRays/s", "cores": threads, "kind": "port",
           "sample": f"{n_views} of {w.n_view} views evenly spaced ({n} rays, {dt:.1f} s fwd+adj), "
                     "extrapolated linearly (rays are independent)"}
    if gpu_view0 is not None and case.vol.ndim == 3:
        f_gpu, a_gpu, y0 = (np.asarray(a, dtype=np.float64) for a in gpu_view0)
        pv = case.per_view
        s64, d64 = case.src[:pv].astype(np.float64), case.dst[:pv].astype(np.float64)
        Mi64, b64 = np.linalg.inv(case.M), case.b.astype(np.float64)
        f64 = O.fwd_planesort(case.vol, Mi64, b64, s64, d64, dtype=np.float64)
        a64 = O.back_planesort(y0, Mi64, b64, s64, d64, case.vol.shape, dtype=np.float64)

        # the reference's own float32 arithmetic: the oracle's restatement of
        # its on-the-fly kernel (ct_projector_3d.cu:902-1012)
        f32 = O.fwd_planesort(case.vol, case.Mi, case.b, case.src[:pv], case.dst[:pv])
        a32 = O.back_planesort(y0.astype(np.float32), case.Mi, case.b, case.src[:pv], case.dst[:pv],
                               case.vol.shape)

        def errs(a, ref):
            return {"max_rel": float(np.abs(a - ref).max() / np.abs(ref).max()),
                    "rel_l2": float(np.linalg.norm(a - ref) / np.linalg.norm(ref))}
        out["view_check"] = {"rays": pv, "view": 0,
                             "vs_reference_f32": {"forward": errs(f_gpu, f32), "adjoint": errs(a_gpu, a32)},
                             "vs_fp64": {"forward": errs(f_gpu, f64), "adjoint": errs(a_gpu, a64)}}
    return out


def _workloads_standalone():
    """workloads.py loaded by file path: the reference arm builds its rays and
    phantom from the package's self-contained geometry and phantom files
    without importing the package, so the only native libraries this process
    maps are the oracle's."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_ctlab_workloads",
                                                  os.path.join(ROOT, "ct_laboratory_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod  # (dataclasses look their module up there)
    spec.loader.exec_module(mod)
    return mod.WORKLOADS


def run_reference(args, world, rank):
    """The reference's CPU projector on this host's cores (rank 0 only)."""
    if rank != 0:
        return
    w = _workloads_standalone().get(args.workload)
    if w is None or not w.name.startswith(("cone", "fan")):
        print(json.dumps({"impl": "reference", "unavailable": f"the reference CPU arm covers the cone-beam and "
                                                              f"fan-beam workloads, not {args.workload}"}))
        return
    case = CpuCase(w)
    threads = cpu_threads()
    rate, _, _ = case.rate([0], threads)
    n_views = int(max(1, min(w.n_view, math.floor(args.ref_step_s * rate / case.per_view))))
    for i in range(args.warmup):
        case.rate([i % w.n_view], threads)
    rays, secs = 0, 0.0
    for k in range(args.steps):
        vs = [(k * 7 + j * max(1, w.n_view // n_views)) % w.n_view for j in range(n_views)]
        r, n, dt = case.rate(vs, threads)
        rays += n
        secs += dt
    value = rays / secs / 1e9
    out = {"metric": METRIC, "value": value, "unit": "GRays/s", "impl": "reference", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": w.name, "n_ray": w.n_ray, "sample_views_per_step": n_views},
           "cpu_baseline": {"value": value, "unit": "GRays/s", "cores": threads, "kind": "port",
                            "sample": f"{n_views} views per step of {w.n_view}, rotating"},
           "e2e": {"value": value, "unit": "GRays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    assert "ct_laboratory_b200" not in sys.modules, "the reference arm must not import the package"
    print(json.dumps(out))


# --------------------------------------------------------------------------- GPU leg
def run_ours(args, world, rank, local):
    from ct_laboratory_b200 import ConeBeam3DProjector, FanBeam2DProjector
    import dataclasses

    from ct_laboratory_b200.workloads import WORKLOADS
    w = WORKLOADS[args.workload]
    if args.views:
        w = dataclasses.replace(w, n_view=args.views, name=f"{w.name}-v{args.views}")
    dev = torch.device("cuda", local)
    if w.name.startswith("cone"):
        proj = ConeBeam3DProjector(*w.n, n_view=w.n_view, det_nx=w.det_nx, det_ny=w.det_ny, sid=w.sid, sdd=w.sdd,
                                   det_spacing=w.pitch, voxel_size=w.voxel, device=dev, tile_rows=args.tile_rows,
                                   voxel_rule=args.voxel_rule, walk=args.walk,
                                   deterministic_adjoint=args.deterministic, block_threads=args.block_threads)
    elif w.name.startswith("static"):
        # StaticCT ring: the modules' 16-row columns take the column walk
        proj = w.projector(dev, voxel_rule=args.voxel_rule, deterministic_adjoint=args.deterministic or False)
    else:
        proj = FanBeam2DProjector(*w.n, n_view=w.n_view, n_det=w.n_det, sid=w.sid, sdd=w.sdd, det_spacing=w.pitch,
                                  pixel_size=w.pixel, device=dev)
    n_ray = proj.src.shape[0]
    shard = (0, n_ray)
    base = proj  # the whole scan's projector (the CPU and MAP legs use it)
    if args.sharded:
        # one scan, its views split across the ranks: all-gather of the
        # sinogram shards (forward), all-reduce of the partial volumes (adjoint)
        from ct_laboratory_b200.sharded import RaySharded3DProjector
        proj = RaySharded3DProjector(proj)
        shard = (proj.lo, proj.hi)
    rays_per_step = n_ray if args.sharded else world * n_ray  # the whole job's rays
    x = w.phantom(device=dev)
    y = torch.rand(n_ray, device=dev, generator=torch.Generator(device=dev).manual_seed(1))
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    # our kernels per step: the forward walk, then the adjoint's -- one walk
    # (atomic scatter); ray table + gather; or max|y|, scale, walk, convert
    launches_per_step = 1 + {None: 1, "gather": 2, "fixed": 4}[args.deterministic]

    def fwd():
        return _fwd3(proj, x) if w.name.startswith(("cone", "static")) else proj.forward_project(x)

    def adj():
        return proj.back_project(y)

    with torch.no_grad():
        for _ in range(args.warmup):
            fwd()
            adj()
        torch.cuda.synchronize(dev)
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
        barrier(world)
        torch.cuda.synchronize(dev)
        with ClockSampler(local) as clk:
            for k in range(args.steps):
                flush.zero_()
                ev[k][0].record(stream)
                fwd()
                ev[k][1].record(stream)
                adj()
                ev[k][2].record(stream)
            torch.cuda.synchronize(dev)
        barrier(world)
    t_fwd = np.array([e[0].elapsed_time(e[1]) for e in ev])
    t_adj = np.array([e[1].elapsed_time(e[2]) for e in ev])
    total_ms = float((t_fwd + t_adj).sum())
    total_ms = max_over_ranks(total_ms, world)
    value = rays_per_step * args.steps / (total_ms / 1e3) / 1e9

    # the launches cover the scan's active tiles (CTProjector3DModule.active_tiling_for)
    tiles_note = "every tile"
    local = getattr(proj, "local", proj)
    if hasattr(local, "_launch_tiling"):
        t = local._launch_tiling()
        act = getattr(t, "active", None)
        if act is not None:
            from ct_laboratory_b200 import _native as N
            n_all = int(N.lib.ctlab_tile_count(int(local.src.shape[0]), N.tiling_ref(t)))
            tiles_note = f"active tiles only: {act[1]} of {n_all} (the rest hold no ray that crosses the volume)"
    peak, peak_src = peaks()
    bytes_per_launch, seg = algorithmic_bytes(w.name, n_ray)
    if args.sharded and bytes_per_launch:
        # this rank's share of the scan's bytes (views carry nearly equal
        # segment counts); its launch times include the collectives
        bytes_per_launch = bytes_per_launch * (shard[1] - shard[0]) / n_ray
    kern = {}
    for name, t in (("forward", t_fwd), ("adjoint", t_adj)):
        ms = float(t.mean())
        ach = bytes_per_launch / (ms / 1e3) / 1e9 if bytes_per_launch else None
        kern[name] = {"ms_mean": ms, "ms_min": float(t.min()), "achieved_gbs": ach,
                      "frac": (ach / peak) if ach else None}
    dom = max(kern, key=lambda k: kern[k]["ms_mean"])
    traffic = load_traffic(w.name, dom, args.voxel_rule)
    roofline = {"bound": "hbm", "achieved": kern[dom]["achieved_gbs"], "peak": peak, "unit": "GB/s",
                "frac": kern[dom]["frac"], "traffic": traffic, "kernel": dom, "peak_source": peak_src,
                "algorithmic_bytes_per_launch": bytes_per_launch, "segments": seg, "kernels": kern}

    e2e = run_e2e(proj, x, y, args, dev, w, world, rays_per_step) if args.e2e_steps > 0 else None
    batched = run_batched(args, dev, flush) if (world == 1 and args.batched_steps > 0) else None
    serving = run_serving(args, dev) if (world == 1 and args.serve_jobs > 0) else None
    map_leg = run_map(args, dev, base, x, y) if (world == 1 and args.map_iters > 0 and w.name.startswith("cone")) \
        else None
    cpu = None
    if world == 1 and rank == 0 and args.cpu_baseline_s > 0:
        view0 = None
        if w.name.startswith(("cone", "static")):
            pv = w.n_ray // w.n_view
            with torch.no_grad():
                y0 = torch.zeros_like(y)
                y0[:pv] = y[:pv]
                view0 = (base.forward_project(x)[:pv].cpu().numpy(), base.back_project(y0).cpu().numpy(),
                         y[:pv].cpu().numpy())
        cpu = cpu_baseline(CpuCase(w, base.src, base.dst, base.M, base.b, x), args.cpu_baseline_s, view0)
    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": "GRays/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
               "scaling": "strong" if args.sharded else "weak", "vs_baseline": None, "dtype": "f32",
               "data": "synthetic",
               "config": {"workload": w.name, "n_ray": n_ray, "volume": list(w.n),
                          "views": w.n_view, "rays_per_rank": shard[1] - shard[0],
                          "l2": "flushed (512 MiB write) before each step",
                          "tile_rows": args.tile_rows, "block_threads": args.block_threads,
                          "voxel_rule": ["midpoint", "crossing"][args.voxel_rule],
                          "walk": ["auto", "lane", "column"][args.walk],
                          "tiles": tiles_note,
                          "adjoint": {None: "float atomic scatter", "gather": "voxel gather (reproducible)",
                                      "fixed": "64-bit fixed-point scatter (reproducible)"}[args.deterministic],
                          "parallelism": (f"ray-sharded x{world}: one scan, whole views per rank, NCCL "
                                          "all-gather (forward) and all-reduce (adjoint)") if args.sharded
                          else f"independent scans x{world}"},
               "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk.summary(), "batched": batched,
               "serving": serving, "map": map_leg,
               "gpu_launches": launches_per_step * args.steps}
        if cpu is not None and "view_check" in cpu:
            out["parity"] = dict(cpu["view_check"], bar=1e-5, metric="max |ours - ref| / max |ref|",
                                 note="view 0 of the benched projector (same kernels, same launch shape) against "
                                      "the CPU restatement of the reference's float32 on-the-fly kernel and against "
                                      "its float64 evaluation")
        print(json.dumps(out))


def _fwd3(proj, x):
    return proj.forward_project(x)


def run_e2e(proj, x, y, args, dev, w, world=1, rays_per_step=None):
    """Public API, host buffers: H2D of the volume and of the adjoint input,
    D2H of the sinogram and of the back-projection, every step.  The device
    inputs are double-buffered and each copy direction has its own stream
    (PCIe is full duplex, and the GPU has a copy engine per direction), so
    step i+1's inputs upload while step i computes and step i's results
    download under step i+1; the timed region ends when every copy of the
    last step has landed.

    Ray-sharded (one scan over the ranks): every rank uploads the volume and
    its own shard of the adjoint input, and downloads its own shard of the
    all-gathered sinogram; rank 0 downloads the summed back-projection.  So
    the job's sinograms cross the host links once in all, while the device
    work is what the device-timed value measures."""
    import torch.distributed as dist
    sharded = bool(getattr(args, "sharded", False)) and hasattr(proj, "lo")
    rank = dist.get_rank() if (sharded and dist.is_initialized()) else 0
    lo, hi = (proj.lo, proj.hi) if sharded else (0, y.numel())
    x_h = x.cpu().pin_memory()
    y_h = y[lo:hi].cpu().pin_memory()
    sino_h = torch.empty(hi - lo, dtype=torch.float32).pin_memory()
    get_vol = rank == 0 or not sharded
    vol_h = torch.empty(x.shape if get_vol else (0,), dtype=torch.float32).pin_memory()
    xd = [torch.empty_like(x) for _ in range(2)]
    yd = [torch.empty(hi - lo, dtype=y.dtype, device=y.device) for _ in range(2)]
    stream = torch.cuda.current_stream(dev)
    h2d, d2h = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    done = [None, None]  # compute of the step that last used buffer set k
    it = [0]

    def step():
        k = it[0] % 2
        it[0] += 1
        with torch.cuda.stream(h2d):
            if done[k] is not None:
                h2d.wait_event(done[k])  # that step is done with xd[k] / yd[k]
            xd[k].copy_(x_h, non_blocking=True)
            ev_x = h2d.record_event()
            yd[k].copy_(y_h, non_blocking=True)
            ev_y = h2d.record_event()
        stream.wait_event(ev_x)
        s = proj(xd[k])
        ev_f = stream.record_event()
        stream.wait_event(ev_y)
        v = proj.back_project(yd[k])
        ev_b = stream.record_event()
        done[k] = ev_b
        with torch.cuda.stream(d2h):
            d2h.wait_event(ev_f)
            sino_h.copy_(s.reshape(-1)[lo:hi], non_blocking=True)
            s.record_stream(d2h)
            d2h.wait_event(ev_b)
            if get_vol:
                vol_h.copy_(v, non_blocking=True)
            v.record_stream(d2h)

    with torch.no_grad():
        for _ in range(2):
            step()
        torch.cuda.synchronize(dev)
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.e2e_steps):
            step()
        stream.wait_stream(d2h)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        barrier(world)
    # the job's time is the slowest rank's
    ms = max_over_ranks(e0.elapsed_time(e1), world) / args.e2e_steps
    n_ray = y.numel()
    rays = world * n_ray if rays_per_step is None else rays_per_step
    if sharded:  # the job's bytes: every rank's volume upload, one sinogram each way, one volume back
        h2d = world * x_h.numel() * 4 + n_ray * 4
        d2h = n_ray * 4 + x.numel() * 4
    else:
        h2d = world * (x_h.numel() * 4 + y_h.numel() * 4)
        d2h = world * (sino_h.numel() * 4 + vol_h.numel() * 4)
    return {"value": rays / (ms / 1e3) / 1e9, "unit": "GRays/s", "ms_per_step": ms,
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "api": f"{type(proj).__name__}.__call__ + .back_project" +
                   ", inputs double-buffered, H2D and D2H each on a stream of its own"}


def run_batched(args, dev, flush):
    """64 uneven 2-D scans (batch64): forward + adjoint of every scan in one
    persistent launch each (autotuned tile shape), replayed from a CUDA graph,
    against the per-scan loop of the same kernels.  Inputs resident, L2
    flushed before every pass."""
    from ct_laboratory_b200.batched import ScanBatch
    from ct_laboratory_b200.workloads import WORKLOADS
    w = WORKLOADS["batch64"]
    t0 = time.perf_counter()
    batch = ScanBatch(w.projectors(dev))
    for img, ph in zip(batch.images_in, w.phantoms(device=dev)):
        img.copy_(ph)
    g = torch.Generator(device=dev).manual_seed(2)
    for s in batch.sinos_in:
        s.copy_(torch.rand(s.shape, generator=g, device=dev))
    setup_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    cfg = batch.autotune(reps=3)
    tune_s = time.perf_counter() - t0
    graph = batch.capture()
    stream = torch.cuda.current_stream(dev)

    def timed(fn):
        fn()
        torch.cuda.synchronize(dev)
        ts = []
        for _ in range(args.batched_steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize(dev)
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    with torch.no_grad():
        ms_graph = timed(graph.replay)
        ms_eager = timed(lambda: (batch.forward(), batch.back()))
        ms_loop = timed(lambda: (batch.forward_loop(), batch.back_loop()))
    n_ray = sum(int(p.src.shape[0]) for p in batch.projectors)
    bytes_pair = 2 * (4 * SEGMENTS["batch64"] + 4 * n_ray)
    # kernels per pass.  Persistent: forward 1; adjoint zeroing, walk and (2-D)
    # the add-back of the transposed scratch.  Loop: one launch per scan and
    # direction, plus one add-back per 2-D scan.
    n_scan, tr = len(batch.projectors), int(batch.scratch is not None)
    per_fwd = {"persistent": 1, "loop": n_scan}
    per_adj = {"persistent": 2 + tr, "loop": n_scan * (1 + tr)}
    launches_graph = per_fwd[cfg["mode"]] + per_adj[batch.config_adj["mode"]]
    launches_loop = per_fwd["loop"] + per_adj["loop"]
    peak, _ = peaks()
    del graph
    return {"workload": "batch64", "n_scan": len(batch.projectors), "n_ray": n_ray, "segments": SEGMENTS["batch64"],
            "tile": {"forward": {k: cfg[k] for k in ("block_threads", "kind", "n_cta", "mode")},
                     "adjoint": {k: batch.config_adj[k] for k in ("block_threads", "kind", "n_cta", "mode")}},
            "ms_per_pass": {"graph": ms_graph, "batched": ms_eager, "per_scan_loop": ms_loop},
            "grays_s": {"graph": n_ray / ms_graph / 1e6, "batched": n_ray / ms_eager / 1e6,
                        "per_scan_loop": n_ray / ms_loop / 1e6},
            "speedup_vs_loop": ms_loop / ms_graph, "gpu_launches_per_pass": {"graph": launches_graph, "per_scan_loop": launches_loop},
            "roofline_frac": bytes_pair / (ms_graph / 1e3) / 1e9 / peak,
            "setup_s": setup_s, "autotune_s": tune_s,
            "note": "one pass = forward + adjoint of all 64 scans; L2 flushed before each pass; median of "
                    f"{args.batched_steps}"}


def run_serving(args, dev):
    """MAP reconstruction jobs arriving as a Poisson process (serve workload):
    the plain per-job loop (reference-style estimator, one job at a time)
    and the continuous-batching server on the same requests, back to back.
    Latency = wall time from a job's arrival to its reconstruction on the
    host; throughput = jobs / (last finish - first arrival)."""
    import dataclasses

    from ct_laboratory_b200.serving import ReconServer, latency_summary, make_jobs, sequential_baseline
    from ct_laboratory_b200.workloads import WORKLOADS
    w = dataclasses.replace(WORKLOADS["serve"], n_jobs=args.serve_jobs)
    t0 = time.perf_counter()
    jobs = make_jobs(w, dev)
    make_s = time.perf_counter() - t0
    plain = sequential_baseline(jobs, dev)
    sa = None
    if args.serve_policy_all:
        server_all = ReconServer(dev, policy="all")
        sa = latency_summary(server_all.run(jobs))
    server = ReconServer(dev, policy="srpt")
    served = server.run(jobs)
    ps, ss = latency_summary(plain), latency_summary(served)
    # the projector work every schedule on this GPU must do: each job's
    # iterations x its measured forward + adjoint pair
    work_s = sum(j.iters * j.pair_ms for j in jobs) / 1e3
    geo = {}
    for j in jobs:
        geo[(j.n, j.views)] = geo.get((j.n, j.views), 0) + 1
    xs = {r["job_id"]: r["x"] for r in served}
    rel = []
    for r in plain:
        a, b = xs[r["job_id"]].double(), r["x"].double()
        rel.append(float((a - b).norm() / b.norm().clamp_min(1e-30)))
    mix = {}
    for j in jobs:
        mix[j.n] = mix.get(j.n, 0) + 1
    return {"workload": "serve", "jobs": len(jobs), "arrival_rate_per_s": w.rate,
            "mix": {f"{k}^3": v for k, v in sorted(mix.items())},
            "rays_x_iters": sum(j.n_ray * j.iters for j in jobs),
            "plain_loop": ps, "served": ss, "served_all_every_tick": sa,
            "throughput_ratio": ss["jobs_per_s"] / ps["jobs_per_s"],
            "projector_work_s": work_s,
            "throughput_ratio_bound": ps["makespan_s"] / work_s,
            "served_breakdown_s": {"projector_launches": server.log[-1]["projector_s"],
                                   "per_job_elementwise": server.log[-1]["elementwise_s"],
                                   "host_and_idle": ss["makespan_s"] - server.log[-1]["projector_s"]
                                   - server.log[-1]["elementwise_s"]},
            "jobs_sharing_a_geometry": sum(c for c in geo.values() if c > 1),
            "p50_ratio": ss["p50_s"] / ps["p50_s"], "p99_ratio": ss["p99_s"] / ps["p99_s"],
            "max_rel_rmse_served_vs_plain": max(rel),
            "served_max_active": server.log[-1]["max_active"], "served_ticks": server.log[-1]["ticks"],
            "request_build_s": make_s,
            "note": "plain loop = ConeBeam3DProjector + MaximumAPosterioriEstimator per job in arrival order; "
                    "served = ReconServer, policy srpt (admission by HBM budget; each tick one batched forward and "
                    "adjoint launch over the active jobs with the least remaining work, >= 64M rays); "
                    "served_all_every_tick = the same server advancing every active job each tick "
                    "(--serve-policy-all); projector_work_s = sum over jobs of iterations x one measured forward + "
                    "adjoint pair of the job's scan, so throughput_ratio_bound = plain makespan / that work bounds "
                    "any schedule of these projector calls on this GPU; jobs_sharing_a_geometry = jobs whose "
                    "(volume, views) another job also has (only those could share one multi-volume walk)"}


def run_map(args, dev, proj, x_true, y_rand):
    """MAP reconstruction on the benchmark scan (cone256): Poisson counts at
    I0 = 1e5 (seeded), quadratic smoothness prior weight 1e-2, a k = 64
    sparse-eigen preconditioner of G = A^T A by Lanczos (every matvec one
    forward + adjoint pass), then 50 preconditioned gradient steps through the
    autograd Function; the gradient checked by central differences (step
    1e-3) at 16 seeded voxels, and the adjoint identity <Ax, y> = <x, A^T y>
    at full size."""
    from ct_laboratory_b200.bayesian_estimation import MaximumAPosterioriEstimator
    from ct_laboratory_b200.random_variable import BeerLambertPoissonRandomVariable, QuadraticSmoothnessRandomVariable
    from ct_laboratory_b200.sparse_eigen_preconditioner import SparseEigenDecomposition
    I0, w_prior, h = 1e5, 1e-2, 1e-3
    out = {"I0": I0, "prior_weight": w_prior}
    with torch.no_grad():
        ax = proj.forward_project(x_true)
        aty = proj.back_project(y_rand)
        lhs = float(torch.dot(ax.double().reshape(-1), y_rand.double().reshape(-1)))
        rhs = float(torch.dot(x_true.double().reshape(-1), aty.double().reshape(-1)))
        out["adjoint_identity_rel"] = abs(lhs - rhs) / abs(lhs)
        g = torch.Generator(device=dev).manual_seed(7)
        counts = torch.poisson(I0 * torch.exp(-ax), generator=g)
        del aty
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    dec = SparseEigenDecomposition(proj, k=args.map_k, volume_shape=tuple(x_true.shape))
    dec.compute_weights(method="lanczos", compute_projection_basis=False, max_restarts=args.lanczos_restarts)
    torch.cuda.synchronize(dev)
    lz_s = time.perf_counter() - t0
    ev = dec.eigenvalues
    out["lanczos"] = {"k": args.map_k, "matvecs": dec.n_matvec, "seconds": lz_s,
                      "ms_per_matvec": 1e3 * lz_s / max(dec.n_matvec, 1), "eig_max": float(ev[0]),
                      "eig_k": float(ev[-1]), "max_restarts": args.lanczos_restarts}
    P = dec.to_image_preconditioner()
    del dec
    lik = BeerLambertPoissonRandomVariable(op=proj.forward_project, I0=I0)
    prior = QuadraticSmoothnessRandomVariable(weight=w_prior)
    est = MaximumAPosterioriEstimator(lik, prior, measurements=counts, x_init=torch.zeros_like(x_true),
                                      preconditioner=P, lr=1.0 / I0)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    xr = est.estimate(num_iters=args.map_iters)
    torch.cuda.synchronize(dev)
    map_s = time.perf_counter() - t0
    rel_true = float((xr - x_true).double().norm() / x_true.double().norm())
    out["map"] = {"iters": args.map_iters, "seconds": map_s, "ms_per_iter": 1e3 * map_s / args.map_iters,
                  "loss_first": est.history[0][0], "loss_last": est.history[-1][0], "rel_err_vs_phantom": rel_true}
    # gradient check at the estimate: autograd (hand-written adjoint) vs central differences
    xv = xr.detach().clone().requires_grad_(True)
    loss, _, _ = est.negative_log_posterior(xv)
    loss.backward()
    grad = xv.grad.detach()
    yd = counts.double()

    def nll_terms(p):  # per-ray Poisson terms in double (lgamma(y + 1) cancels in differences)
        rate = I0 * torch.exp(-p.double())
        return rate - yd * torch.log(rate)

    def prior_energy(v):
        return sum(float(torch.diff(v.double(), dim=d).pow(2).sum()) for d in range(3)) * 0.5 * w_prior

    gen = np.random.default_rng(11)
    vox = [tuple(int(gen.integers(64, 192)) for _ in range(3)) for _ in range(16)]
    errs = []
    with torch.no_grad():
        base = xr.detach().clone()
        for v in vox:
            xp, xm = base.clone(), base.clone()
            xp[v] += h
            xm[v] -= h
            d_nll = float((nll_terms(proj.forward_project(xp)) - nll_terms(proj.forward_project(xm))).sum())
            # the prior changes only around v: difference of its energies in double
            sl = tuple(slice(max(c - 2, 0), c + 3) for c in v)
            d_pr = prior_energy(xp[sl]) - prior_energy(xm[sl])
            fd = (d_nll + d_pr) / (2 * h)
            errs.append(abs(fd - float(grad[v])) / max(abs(float(grad[v])), 1e-30))
    out["finite_differences"] = {"voxels": len(vox), "step": h, "max_rel_err": max(errs),
                                 "median_rel_err": float(np.median(errs))}
    return out


def load_traffic(workload, kernel, voxel_rule=0):
    """DRAM bytes per launch from the committed ncu summary, if any (keyed
    by workload, and "<workload>/crossing" for the crossing voxel rule)."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    return d.get(workload if voxel_rule == 0 else f"{workload}/crossing", {}).get(kernel)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="cone256")
    ap.add_argument("--tile-rows", type=int, default=32)
    ap.add_argument("--block-threads", type=int, default=128, help="threads per CTA of the cone-beam launches")
    ap.add_argument("--voxel-rule", type=int, default=0, help="0 = reference midpoint rule, 1 = crossing rule")
    ap.add_argument("--walk", type=int, default=0, help="0 = auto, 1 = per-lane walk, 2 = column walk")
    ap.add_argument("--deterministic", nargs="?", const="fixed", default=None, choices=["fixed", "gather"],
                    help="reproducible adjoint: 'fixed' (default; the forward's walk scattering in 64-bit fixed "
                         "point) or 'gather' (voxel-driven, crossing rule)")
    ap.add_argument("--sharded", action="store_true",
                    help="split one scan's views across the ranks (the default when N > 1; with N = 1 the "
                         "same path over a one-rank group)")
    ap.add_argument("--replicas", action="store_true", help="N > 1: every rank projects its own whole scan")
    ap.add_argument("--views", type=int, default=0,
                    help="override the workload's view count (smaller cases for profiler captures)")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--map-iters", type=int, default=50, help="MAP iterations on the cone scan (0 = skip the leg)")
    ap.add_argument("--map-k", type=int, default=64, help="eigenpairs of the Lanczos preconditioner")
    ap.add_argument("--lanczos-restarts", type=int, default=8)
    ap.add_argument("--serve-jobs", type=int, default=100,
                    help="jobs of the MAP serving workload (0 = skip that leg)")
    ap.add_argument("--serve-policy-all", action="store_true",
                    help="also serve with every active job advancing each tick")
    ap.add_argument("--batched-steps", type=int, default=10,
                    help="timed passes of the 64-scan batched workload (0 = skip that leg)")
    ap.add_argument("--cpu-baseline-s", type=float, default=15.0)
    ap.add_argument("--ref-step-s", type=float, default=4.0)
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if int(os.environ.get("WORLD_SIZE", "1")) > 1 and not args.replicas and not args.workload.startswith("fan"):
        args.sharded = True
    if args.workload.startswith("fan"):
        args.sharded = False  # the ray-sharded projector is 3-D
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1 or (args.sharded and args.impl == "ours"):
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
