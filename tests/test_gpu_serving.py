"""Continuous-batching MAP serving (ReconServer) against the plain per-job
loop through the reference-style API, alone-vs-mixed invariance, admission
by HBM budget and mid-run joins.

Tolerance: reconstructions within 1e-4 relative RMSE (the stated MAP bar)
of the sequential MaximumAPosterioriEstimator run and of the same job
served alone; the server's iteration is written out instead of autograd and
its adjoint adds in a different atomic order, so results agree to float
rounding, not bitwise -- except with the fixed-point adjoint
(deterministic_adjoint=True), where a job alone and in the mix agree
bitwise."""
import dataclasses

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")
TOL = 1e-4


def small_workload(**kw):
    from ct_laboratory_b200.workloads import ServingWorkload
    args = dict(n_jobs=5, rate=200.0, sizes=(24, 32, 40), probs=(0.4, 0.3, 0.3), views=(12, 30), iters=(5, 10),
                I0=(1e4, 1e5), seed=3)
    args.update(kw)
    return ServingWorkload(**args)


def rel_rmse(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.fixture(scope="module")
def jobs():
    from ct_laboratory_b200.serving import make_jobs
    return make_jobs(small_workload(), DEV)


def test_served_matches_sequential_estimator(jobs):
    from ct_laboratory_b200.serving import ReconServer, sequential_baseline
    served = {r["job_id"]: r for r in ReconServer(DEV).run(jobs)}
    plain = {r["job_id"]: r for r in sequential_baseline(jobs, DEV)}
    for j in jobs:
        s, p = served[j.job_id], plain[j.job_id]
        assert s["iters"] == p["iters"] == j.iters
        assert float(p["x"].abs().max()) > 0
        assert rel_rmse(s["x"], p["x"]) <= TOL, (j.job_id, rel_rmse(s["x"], p["x"]))


def test_result_same_alone_and_in_the_mix(jobs):
    from ct_laboratory_b200.serving import ReconServer
    mixed = {r["job_id"]: r["x"] for r in ReconServer(DEV).run(jobs)}
    for j in jobs:
        alone = ReconServer(DEV).run([dataclasses.replace(j, arrival_s=0.0)])[0]["x"]
        assert rel_rmse(mixed[j.job_id], alone) <= TOL, j.job_id


def test_admission_respects_the_hbm_budget(jobs):
    from ct_laboratory_b200.serving import ReconServer, job_bytes
    big = sorted(job_bytes(j) for j in jobs)
    budget = big[-1] + big[-2]  # room for the two largest at once, never three
    server = ReconServer(DEV, budget_bytes=budget)
    out = server.run([dataclasses.replace(j, arrival_s=0.0) for j in jobs])
    assert len(out) == len(jobs) and all("x" in r for r in out)
    assert 1 <= server.log[-1]["max_active"] <= 2
    one = ReconServer(DEV, max_active=1)
    one.run(jobs)
    assert one.log[-1]["max_active"] == 1


def test_late_arrival_joins_running_jobs(jobs):
    from ct_laboratory_b200.serving import ReconServer
    early = dataclasses.replace(jobs[0], arrival_s=0.0, iters=3000)
    late = dataclasses.replace(jobs[1], arrival_s=0.002)
    for policy in ("all", "srpt"):
        server = ReconServer(DEV, policy=policy)
        res = {r["job_id"]: r for r in server.run([early, late])}
        # the late job is admitted while the early one is still iterating
        assert res[late.job_id]["admit_s"] < res[early.job_id]["finish_s"], policy
        assert server.log[-1]["max_active"] == 2
        if policy == "srpt":  # the short late job overtakes the long one
            assert res[late.job_id]["finish_s"] < res[early.job_id]["finish_s"]


def test_srpt_and_all_policies_give_the_same_reconstructions(jobs):
    from ct_laboratory_b200.serving import ReconServer
    a = {r["job_id"]: r["x"] for r in ReconServer(DEV, policy="all").run(jobs)}
    b = {r["job_id"]: r["x"] for r in ReconServer(DEV, policy="srpt", tick_rays=1).run(jobs)}
    for j in jobs:
        assert rel_rmse(a[j.job_id], b[j.job_id]) <= TOL


def test_deterministic_adjoint_alone_and_in_the_mix_bitwise(jobs):
    """With the fixed-point adjoint a job's reconstruction is the same bits
    served alone, among the others, and under either scheduling policy; and
    it stays within the MAP bar of the float-atomic server."""
    from ct_laboratory_b200.serving import ReconServer
    mixed = {r["job_id"]: r["x"] for r in ReconServer(DEV, deterministic_adjoint=True).run(jobs)}
    srpt = {r["job_id"]: r["x"] for r in ReconServer(DEV, deterministic_adjoint=True, policy="srpt",
                                                      tick_rays=1).run(jobs)}
    atomic = {r["job_id"]: r["x"] for r in ReconServer(DEV).run(jobs)}
    for j in jobs:
        alone = ReconServer(DEV, deterministic_adjoint=True).run([dataclasses.replace(j, arrival_s=0.0)])[0]["x"]
        assert torch.equal(mixed[j.job_id], alone), j.job_id
        assert torch.equal(mixed[j.job_id], srpt[j.job_id]), j.job_id
        assert rel_rmse(mixed[j.job_id], atomic[j.job_id]) <= TOL, j.job_id


def test_scan_batch_deterministic_adjoint_is_scan_independent():
    """ScanBatch(deterministic_adjoint=True): each scan's adjoint is the same
    bits in any batch and equals the single-scan fixed-point call."""
    from ct_laboratory_b200 import ConeBeam3DProjector
    from ct_laboratory_b200.batched import ScanBatch
    from ct_laboratory_b200.tomography import back_project_3d_fixed_cuda
    ps = [ConeBeam3DProjector(n, n, n, n_view=v, det_nx=40, det_ny=32, sid=100.0, sdd=150.0, det_spacing=0.8,
                              voxel_size=0.5, voxel_rule=1, device=DEV) for n, v in ((24, 10), (32, 7), (20, 12))]
    g = torch.Generator(device=DEV).manual_seed(4)
    ys = [torch.rand(p.src.shape[0], generator=g, device=DEV) for p in ps]
    outs = []
    for sel in ([0, 1, 2], [1], [2, 0]):
        b = ScanBatch([ps[i] for i in sel], deterministic_adjoint=True)
        for k, i in enumerate(sel):
            b.sinos_in[k].copy_(ys[i])
        b.back()
        outs.append({i: b.images_out[k].clone() for k, i in enumerate(sel)})
    for i, p in enumerate(ps):
        want = back_project_3d_fixed_cuda(ys[i], p.src, p.dst, p.M, p.b, p.n_x, p.n_y, p.n_z, tiling=p.ray_tiling,
                                          M_inv=p.M_inv)
        for o in outs:
            if i in o:
                assert torch.equal(o[i], want), i


def test_native_map_steps_match_the_written_out_iteration():
    """ctlab_map_poisson_residual and ctlab_map_smoothness_step against the
    same iteration written with torch ops (non-periodic differences along
    every axis, including axes of length 1 and 2), to float rounding."""
    from ct_laboratory_b200 import _native as N
    gen = torch.Generator(device=DEV).manual_seed(9)
    for shape in ((5, 7, 3), (1, 4, 6), (2, 1, 9), (16, 16, 16)):
        x = torch.rand(shape, generator=gen, device=DEV)
        grad = torch.rand(shape, generator=gen, device=DEV) - 0.5
        w, lr = 0.3, 0.05
        want_g = grad.clone()
        for d in range(3):
            n = x.shape[d]
            if n > 1:
                diff = torch.diff(x, dim=d)
                want_g.narrow(d, 0, n - 1).sub_(diff, alpha=w)
                want_g.narrow(d, 1, n - 1).add_(diff, alpha=w)
        want_x = x - lr * want_g
        xx, gg = x.clone(), grad.clone()
        N.call("ctlab_map_smoothness_step", N.ptr(xx), N.ptr(gg), *shape, w, lr, N.stream_of(xx))
        assert float((gg - want_g).abs().max()) <= 1e-6 * float(want_g.abs().max()), shape
        assert float((xx - want_x).abs().max()) <= 1e-6 * float(want_x.abs().max()), shape
    p = torch.rand(1000, generator=gen, device=DEV) * 3
    y = torch.poisson(1e4 * torch.exp(-p), generator=gen)
    r = torch.empty_like(p)
    N.call("ctlab_map_poisson_residual", N.ptr(y), N.ptr(p), N.ptr(r), p.numel(), 1e4, N.stream_of(p))
    want = y - 1e4 * torch.exp(-p)
    # (r is a small difference of numbers near I0: compare at the scale of y)
    assert float((r - want).abs().max()) <= 1e-6 * float(y.abs().max())
