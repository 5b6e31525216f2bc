"""Serving MAP reconstruction jobs with continuous batching.

A job is a cone-beam reconstruction request: volume size, number of views,
photon count I0, number of MAP iterations, step size and the measured
counts y (host memory).  ``ReconServer.run(jobs)`` serves a stream of them
as they arrive:

* admission: a job is admitted when it has arrived, a slot is free
  (``max_active``) and its device footprint (geometry, measurements,
  sinogram and volume state, ``job_bytes``) fits the HBM budget next to the
  jobs already running;
* state on the device: an admitted job's geometry, measurements, estimate
  and work buffers stay resident until it finishes;
* continuous batching: every tick runs one MAP iteration of every selected
  job, with one batched forward and one batched adjoint pass over all of
  them (``ScanBatch`` over the jobs' own buffers, uneven sizes and view
  counts: one persistent launch per direction for small scans, one launch
  per scan over its active tiles for scans that fill the GPU alone); the
  Poisson residual, smoothness prior and update are applied per job by
  three fused kernels (ctlab_map_poisson_residual,
  ctlab_map_smoothness_step).  Jobs join and leave between ticks,
  so requests that arrive while others run start as soon as memory and a
  slot free up, and their projector work overlaps with the others' in the
  same launches.

The iteration is the reference's MAP estimator with the identity
preconditioner (bayesian_estimation/map_estimator.py:102-117: loss =
-log p(y|x) - log p(x), one SGD step per iteration) for the Beer-Lambert
Poisson likelihood (probability/random_variables/poisson.py:36-47) and the
non-periodic quadratic smoothness prior (image_energies.py:18-29):

    grad = A^T (y - I0 exp(-A x)) + w * sum_d D_d^T D_d x,     x <- x - lr * grad

written out directly instead of through autograd.  A job's result does not
depend on which other jobs share its launches: the forward is deterministic
and the adjoint differs only in the order of float atomic additions -- with
``deterministic_adjoint=True`` not even that: every job's adjoint scatters
in 64-bit fixed point (integer sums, associative), so a job served alone and
the same job served among others give the same bits.

``sequential_baseline(jobs)`` serves the same jobs one at a time in arrival
order through the reference-style API (``ConeBeam3DProjector`` +
``MaximumAPosterioriEstimator``): the plain per-job loop the server is
measured against.
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native as N
from .batched import ScanBatch
from .tomography import ConeBeam3DProjector

__all__ = ["JobSpec", "ReconServer", "sequential_baseline", "make_jobs", "job_bytes", "latency_summary"]


@dataclass
class JobSpec:
    """One reconstruction request.  `y` holds the measured counts (host,
    ideally pinned), ordered like the scan's rays [view][det_v][det_u]."""
    job_id: int
    arrival_s: float
    n: int
    views: int
    iters: int
    I0: float
    lr: float
    det_nx: int
    det_ny: int
    voxel: float = 0.5
    pitch: float = 0.8
    sid: float = 1000.0
    sdd: float = 1500.0
    prior_w: float = 1e-2
    y: torch.Tensor = field(default=None, repr=False)
    pair_ms: float = 0.0  # one forward + adjoint of this job's scan on the device (make_jobs measures it)

    @property
    def n_ray(self):
        return self.views * self.det_nx * self.det_ny

    def projector(self, device):
        return ConeBeam3DProjector(self.n, self.n, self.n, n_view=self.views, det_nx=self.det_nx,
                                   det_ny=self.det_ny, sid=self.sid, sdd=self.sdd, det_spacing=self.pitch,
                                   voxel_size=self.voxel, voxel_rule=N.VOXEL_CROSSING, device=device,
                                   build_on_device=True)


def job_bytes(spec, deterministic_adjoint=False):
    """Device footprint of an admitted job: rays (src, dst: 24 B), sinograms
    (y, A x, residual: 12 B) per ray; volumes (estimate, gradient and the
    prior's temporaries: 16 B) per voxel; with the fixed-point adjoint also
    its int64 sums (8 B per voxel: the server's one shared workspace is
    sized for the largest job, counted here for every job, an upper
    bound)."""
    return 36 * spec.n_ray + (24 if deterministic_adjoint else 16) * spec.n ** 3


def make_jobs(workload, device, lr_scale=1.0):
    """Requests of a serving workload: for each job a seeded phantom is
    projected, Poisson noise drawn (I0 exp(-A x)) and the counts kept in
    pinned host memory, as a client would send them.  The step size is
    lr_scale / (I0 * max_r (A 1)_r * max_v (A^T 1)_v), the Schur bound on the
    largest eigenvalue of the Poisson Hessian, so that plain gradient steps
    are stable for every job."""
    from .phantoms import ellipsoid_phantom_3d
    jobs = []
    for d in workload.jobs():
        spec = JobSpec(**d)
        p = spec.projector(device)
        x = ellipsoid_phantom_3d(spec.n, spec.n, spec.n, voxel=spec.voxel, n_ellipsoid=8, seed=1000 + spec.job_id,
                                 device=device)
        with torch.no_grad():
            line = p.forward_project(x)
            g = torch.Generator(device=device).manual_seed(2000 + spec.job_id)
            y = torch.poisson(spec.I0 * torch.exp(-line), generator=g)
            row = float(p.forward_project(torch.ones_like(x)).max())
            col = float(p.back_project(torch.ones_like(line)).max())
            # one forward + adjoint pair as an iteration runs it: the adjoint
            # of the first iteration's residual y - I0 exp(-A 0), nonzero on
            # every ray through the volume (the adjoint skips rays whose input
            # is zero, so A x of the phantom would time too little work);
            # the second of two timings
            r0 = y - spec.I0
            for _ in range(2):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                p.forward_project(x)
                p.back_project(r0)
                e1.record()
                e1.synchronize()
            spec.pair_ms = e0.elapsed_time(e1)
            del r0
        spec.lr = lr_scale / (spec.I0 * row * col)
        spec.y = y.cpu().pin_memory()
        jobs.append(spec)
        del p, x, line, y
    torch.cuda.synchronize(device)
    return jobs


class _Active:
    """Device state of an admitted job."""

    def __init__(self, spec, device, deterministic_adjoint=False):
        self.spec = spec
        self.proj = spec.projector(device)
        self.y = spec.y.to(device, non_blocking=True)
        n = spec.n
        self.x = torch.zeros((n, n, n), dtype=torch.float32, device=device)
        self.g = torch.empty_like(self.x)
        self.p = torch.empty(spec.n_ray, dtype=torch.float32, device=device)
        self.r = torch.empty_like(self.p)
        self.it = 0
        self.nbytes = job_bytes(spec, deterministic_adjoint)


def _residual_(job):
    """r = y - I0 exp(-p) into job.r: one pass (ctlab_map_poisson_residual)."""
    N.call("ctlab_map_poisson_residual", N.ptr(job.y), N.ptr(job.p), N.ptr(job.r), job.p.numel(),
           float(job.spec.I0), N.stream_of(job.p))


def _prior_and_step_(job):
    """g += w sum_d D_d^T D_d x (non-periodic differences), then x -= lr g:
    one pass for the prior's gradient, one for the step
    (ctlab_map_smoothness_step)."""
    n = job.spec.n
    N.call("ctlab_map_smoothness_step", N.ptr(job.x), N.ptr(job.g), n, n, n, float(job.spec.prior_w),
           float(job.spec.lr), N.stream_of(job.x))


class ReconServer:
    def __init__(self, device, budget_bytes=None, max_active=16, run_ahead=2, policy="srpt", tick_rays=64_000_000,
                 deterministic_adjoint=False):
        """policy "all": every active job advances one iteration per tick.
        policy "srpt": the active jobs with the least remaining work (rays x
        iterations left) advance, as many as fill `tick_rays` rays per tick
        (at least one): a short job that arrives while long ones run
        overtakes them, and every tick still gives the GPU a full launch."""
        if policy not in ("all", "srpt"):
            raise ValueError(f"unknown policy {policy!r}")
        self.policy = policy
        self.deterministic_adjoint = bool(deterministic_adjoint)
        self.tick_rays = int(tick_rays)
        self.device = torch.device(device)
        if budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            budget_bytes = int(0.7 * free)
        self.budget = int(budget_bytes)
        self.max_active = int(max_active)
        self.run_ahead = int(run_ahead)
        self.log = []

    def _select(self, active):
        if self.policy == "all":
            return list(active)
        order = sorted(active, key=lambda a: (a.spec.n_ray * (a.spec.iters - a.it), a.spec.job_id))
        sel, rays = [], 0
        for a in order:
            if sel and rays >= self.tick_rays:
                break
            sel.append(a)
            rays += a.spec.n_ray
        return sel

    def run(self, jobs, t0=None):
        """Serve `jobs` (arrival_s relative to t0 = now); returns one result
        dict per job: arrival, admission and finish times (s), latency (s),
        the reconstruction (host tensor) and the iterations run."""
        dev = self.device
        queue = deque(sorted(jobs, key=lambda j: j.arrival_s))
        active, finishing, results = [], [], {}
        used = 0
        batch, dirty, batch_key = None, True, None
        det, fixed_ws = self.deterministic_adjoint, None
        ticks = deque()
        n_ticks = peak = 0
        marks = []  # per tick: events before / after the projector and elementwise phases
        t0 = time.perf_counter() if t0 is None else t0
        with torch.no_grad(), torch.cuda.device(dev):
            while queue or active or finishing:
                now = time.perf_counter() - t0
                for f in list(finishing):  # results that reached the host
                    jid, x_dev, host, ev = f
                    if ev.query():
                        results[jid].update(finish_s=time.perf_counter() - t0, x=host)
                        finishing.remove(f)
                while (queue and queue[0].arrival_s <= now and len(active) < self.max_active
                       and used + job_bytes(queue[0], det) <= self.budget):
                    s = queue.popleft()
                    a = _Active(s, dev, det)
                    used += a.nbytes
                    active.append(a)
                    peak = max(peak, len(active))
                    results[s.job_id] = {"job_id": s.job_id, "arrival_s": s.arrival_s,
                                         "admit_s": time.perf_counter() - t0, "iters": s.iters}
                    dirty = True
                if queue and not active and queue[0].arrival_s > now:
                    time.sleep(min(queue[0].arrival_s - now, 0.002))
                    continue
                if queue and not active and used + job_bytes(queue[0], det) > self.budget and not finishing:
                    raise RuntimeError(f"job {queue[0].job_id} needs {job_bytes(queue[0], det)} bytes, more than "
                                       f"the HBM budget {self.budget}")
                if not active:
                    if finishing:
                        torch.cuda.synchronize(dev)
                    continue
                sel = self._select(active)
                key = tuple(id(a) for a in sel)
                if dirty or key != batch_key:
                    if det:  # one int64 workspace for every batch, grown to the largest job
                        need = max(int(N.lib.ctlab_back_project_3d_fixed_workspace_bytes(1, *[a.spec.n] * 3))
                                   for a in sel)
                        if fixed_ws is None or fixed_ws.numel() < need:
                            fixed_ws = None
                            fixed_ws = torch.empty(need, dtype=torch.uint8, device=dev)
                    batch = ScanBatch([a.proj for a in sel], voxel_rule=N.VOXEL_CROSSING,
                                      deterministic_adjoint=det, fixed_workspace=fixed_ws, buffers={"images_in": [a.x for a in sel], "sinos_out": [a.p for a in sel],
                                               "sinos_in": [a.r for a in sel], "images_out": [a.g for a in sel]})
                    batch_key, dirty = key, False
                if len(ticks) >= self.run_ahead:  # bound how far the host runs ahead of the GPU
                    ticks.popleft().synchronize()
                m = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
                m[0].record()
                batch.forward()
                m[1].record()
                for a in sel:
                    _residual_(a)
                m[2].record()
                batch.back()
                m[3].record()
                for a in sel:
                    _prior_and_step_(a)
                    a.it += 1
                m[4].record()
                marks.append(m)
                ev = torch.cuda.Event()
                ev.record()
                ticks.append(ev)
                n_ticks += 1
                done = [a for a in active if a.it >= a.spec.iters]
                if done:
                    batch = None
                    for a in done:
                        host = torch.empty(a.x.shape, dtype=torch.float32, pin_memory=True)
                        host.copy_(a.x, non_blocking=True)
                        fev = torch.cuda.Event()
                        fev.record()
                        # only the estimate stays referenced until its copy has run; the
                        # other buffers go back to the allocator now (their reuse is
                        # ordered after the queued work on this stream)
                        finishing.append((a.spec.job_id, a.x, host, fev))
                        active.remove(a)
                        used -= a.nbytes
                    del a
                    dirty = True
        torch.cuda.synchronize(dev)
        proj_ms = sum(m[0].elapsed_time(m[1]) + m[2].elapsed_time(m[3]) for m in marks)
        elem_ms = sum(m[1].elapsed_time(m[2]) + m[3].elapsed_time(m[4]) for m in marks)
        self.log.append({"ticks": n_ticks, "max_active": peak, "projector_s": proj_ms / 1e3,
                         "elementwise_s": elem_ms / 1e3})
        out = []
        for jid in sorted(results):
            r = results[jid]
            r["latency_s"] = r["finish_s"] - r["arrival_s"]
            out.append(r)
        return out


def sequential_baseline(jobs, device, t0=None):
    """The same jobs one after another in arrival order through the
    reference-style API: ConeBeam3DProjector + BeerLambertPoissonRandomVariable
    + QuadraticSmoothnessRandomVariable + MaximumAPosterioriEstimator
    (identity preconditioner), results read back to the host per job."""
    from .bayesian_estimation import MaximumAPosterioriEstimator
    from .random_variable import BeerLambertPoissonRandomVariable, QuadraticSmoothnessRandomVariable
    dev = torch.device(device)
    t0 = time.perf_counter() if t0 is None else t0
    out = []
    for s in sorted(jobs, key=lambda j: j.arrival_s):
        now = time.perf_counter() - t0
        if s.arrival_s > now:
            time.sleep(s.arrival_s - now)
        start = time.perf_counter() - t0
        p = s.projector(dev)
        y = s.y.to(dev, non_blocking=True)
        lik = BeerLambertPoissonRandomVariable(op=p.forward_project, I0=s.I0)
        prior = QuadraticSmoothnessRandomVariable(weight=s.prior_w)
        est = MaximumAPosterioriEstimator(lik, prior, measurements=y,
                                          x_init=torch.zeros((s.n, s.n, s.n), device=dev), lr=s.lr)
        x = est.estimate(num_iters=s.iters).cpu()
        fin = time.perf_counter() - t0
        out.append({"job_id": s.job_id, "arrival_s": s.arrival_s, "admit_s": start, "finish_s": fin,
                    "latency_s": fin - s.arrival_s, "iters": s.iters, "x": x})
        del p, y, lik, est
    return out


def latency_summary(results):
    lat = np.array([r["latency_s"] for r in results])
    first = min(r["arrival_s"] for r in results)
    last = max(r["finish_s"] for r in results)
    return {"jobs": len(results), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "makespan_s": last - first, "jobs_per_s": len(results) / (last - first)}
