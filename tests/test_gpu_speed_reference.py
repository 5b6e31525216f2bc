"""Speed and full-size parity against the reference's own CUDA projector.

The reference's default cone-beam path is its on-the-fly kernel
(ConeBeam3DProjector defaults to precomputed_intersections=False,
conebeam_projector_3d.py:129; kernel ray_kernel_plane_sort,
src/ct_projector_3d.cu:902-1012), compiled from its sources into oracle/_ref
by oracle/build_ref.py.  Here it runs on an evenly spaced sample of the
views of the cone-beam 256^3 benchmark scan (0.5 mm voxels, 360 views,
512 x 384 cells at 0.8 mm, SID 1000 mm / SDD 1500 mm): its cost per ray is
independent of the other rays, so rays per second on the sample stand for
the whole scan.  Ours runs the whole scan the way the benchmark does
(ConeBeam3DProjector with its defaults: the reference's midpoint voxel rule,
the column walk, 128-thread CTAs; L2 flushed before each pass).

Parity is checked on those full-size views with the benchmark's own launch
shape (the detector tiling of the sampled views) and through the _C entry
points with no launch hint (layout detected), forward and adjoint, and the
reproducible fixed-point adjoint, at the stated 1e-5; the 16-row StaticCT ring (static512) is checked the same way on
a slice of its views.  The reference's adjoint is called through _C with the
correct M^-1 (its Python wrapper would invert twice,
ct_projector_3d_cuda.py:209-210, :319).

Set CTLAB_PERF_OUT=<file> to have the measured figures written as JSON.
"""
import json
import os

import numpy as np
import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu
DEV = "cuda"
SAMPLE_VIEWS = (0, 90, 180, 270)


@pytest.fixture(scope="module")
def ref():
    from oracle.build_ref import load_ref
    mod = load_ref()
    if mod is None:
        pytest.skip("reference CUDA build not present (python oracle/build_ref.py)")
    return mod


def _events_ms(fn, reps, flush=None):
    out = []
    for _ in range(reps):
        if flush is not None:
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        out.append(e0.elapsed_time(e1))
    return float(np.median(out))


def test_cone256_speed_and_parity_vs_reference_cuda(ref):
    from ct_laboratory_b200 import ConeBeam3DProjector, _C
    from ct_laboratory_b200.workloads import WORKLOADS
    w = WORKLOADS["cone256"]
    x = w.phantom(device=DEV)
    proj = ConeBeam3DProjector(*w.n, n_view=w.n_view, det_nx=w.det_nx, det_ny=w.det_ny, sid=w.sid, sdd=w.sdd,
                               det_spacing=w.pitch, voxel_size=w.voxel, device=DEV)
    n_ray = proj.src.shape[0]
    y = torch.rand(n_ray, device=DEV, generator=torch.Generator(device=DEV).manual_seed(1))
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=DEV)
    with torch.no_grad():
        for _ in range(3):
            proj.forward_project(x)
            proj.back_project(y)
        torch.cuda.synchronize()
        t_fwd = _events_ms(lambda: proj.forward_project(x), 5, flush)
        t_adj = _events_ms(lambda: proj.back_project(y), 5, flush)
    ours_rate = n_ray / ((t_fwd + t_adj) / 1e3)
    # the same scan through the bare _C calls the reference's wrappers make
    # (no launch hint, a fresh M^-1 per call)
    with torch.no_grad():
        for _ in range(2):
            _C.forward_project_3d_on_the_fly_cuda(x, proj.src, proj.dst, torch.inverse(proj.M).contiguous(), proj.b)
            _C.back_project_3d_on_the_fly_cuda(y, proj.src, proj.dst, torch.inverse(proj.M).contiguous(), proj.b, *w.n)
        c_fwd = _events_ms(lambda: _C.forward_project_3d_on_the_fly_cuda(x, proj.src, proj.dst,
                                                                         torch.inverse(proj.M).contiguous(), proj.b), 3, flush)
        c_adj = _events_ms(lambda: _C.back_project_3d_on_the_fly_cuda(y, proj.src, proj.dst, torch.inverse(proj.M).contiguous(),
                                                                      proj.b, *w.n), 3, flush)
    c_rate = n_ray / ((c_fwd + c_adj) / 1e3)

    # the sample: whole views, contiguous in the [view][v][u] ray order
    per_view = w.det_nx * w.det_ny
    idx = torch.cat([torch.arange(v * per_view, (v + 1) * per_view, device=DEV) for v in SAMPLE_VIEWS])
    src, dst = proj.src[idx].contiguous(), proj.dst[idx].contiguous()
    ys = y[idx].contiguous()
    Mi = torch.inverse(proj.M).contiguous()
    b = proj.b
    n_s = idx.numel()
    # warm-up on one view, then one timed pass over the sample
    ref.forward_project_3d_on_the_fly_cuda(x, src[:per_view], dst[:per_view], Mi, b)
    ref.back_project_3d_on_the_fly_cuda(ys[:per_view], src[:per_view], dst[:per_view], Mi, b, *w.n)
    torch.cuda.synchronize()
    holder = {}
    r_fwd = _events_ms(lambda: holder.__setitem__("f", ref.forward_project_3d_on_the_fly_cuda(x, src, dst, Mi, b)), 1)
    r_adj = _events_ms(lambda: holder.__setitem__("b", ref.back_project_3d_on_the_fly_cuda(ys, src, dst, Mi, b,
                                                                                            *w.n)), 1)
    ref_rate = n_s / ((r_fwd + r_adj) / 1e3)
    ratio = ours_rate / ref_rate

    # parity at full size on the sampled views: the benchmark's launch shape
    # (its tiling over the sampled views) and the bare _C call
    from ct_laboratory_b200.tomography.conebeam_projector_3d import conebeam_tiling
    til = conebeam_tiling(len(SAMPLE_VIEWS), w.det_nx, w.det_ny, tile_rows=proj.ray_tiling.tile_rows,
                          block_threads=proj.ray_tiling.block_threads, voxel_rule=proj.ray_tiling.voxel_rule)
    rf, rb = holder["f"].cpu().numpy(), holder["b"].cpu().numpy()
    errs = {}
    for name, t in (("bench_tiling", til), ("c_api", None)):
        f = _C.forward_project_3d_on_the_fly_cuda(x, src, dst, Mi, b, tiling=t)
        a = _C.back_project_3d_on_the_fly_cuda(ys, src, dst, Mi, b, *w.n, tiling=t)
        errs[name] = (rel_err(f.cpu().numpy(), rf), rel_err(a.cpu().numpy(), rb))
    # the reproducible (fixed-point) adjoint on the same views and launch shape
    from ct_laboratory_b200.tomography import back_project_3d_fixed_cuda
    fx = back_project_3d_fixed_cuda(ys, src, dst, proj.M, b, *w.n, tiling=til, M_inv=Mi)
    errs["fixed_adjoint"] = (0.0, rel_err(fx.cpu().numpy(), rb.reshape(fx.shape)))
    e_f = max(e[0] for e in errs.values())
    e_b = max(e[1] for e in errs.values())

    res = {"workload": "cone256", "n_ray": n_ray, "ours_ms_fwd": t_fwd, "ours_ms_adj": t_adj,
           "ours_grays_s": ours_rate / 1e9, "c_api_ms_fwd": c_fwd, "c_api_ms_adj": c_adj,
           "c_api_grays_s": c_rate / 1e9, "ref_sample_views": list(SAMPLE_VIEWS), "ref_sample_rays": n_s,
           "ref_ms_fwd_sample": r_fwd, "ref_ms_adj_sample": r_adj, "ref_grays_s": ref_rate / 1e9,
           "ref_ms_fwd_full_extrapolated": r_fwd * n_ray / n_s, "ref_ms_adj_full_extrapolated": r_adj * n_ray / n_s,
           "speedup": ratio, "parity_fwd_rel": e_f, "parity_adj_rel": e_b, "parity_by_path": errs}
    print(json.dumps(res))
    out = os.environ.get("CTLAB_PERF_OUT")
    if out:
        with open(out, "w") as f:
            json.dump(res, f, indent=1)
    assert e_f < 1e-5 and e_b < 1e-5, res
    assert ratio >= 10.0, res


def test_static512_column16_parity_vs_reference_cuda(ref):
    """The StaticCT ring's 16-row modules (two 16-lane groups per warp) under
    the default voxel rule, on four (rotation, source) views of static512,
    against the reference's compiled kernel: forward and adjoint within 1e-5."""
    from ct_laboratory_b200 import _C
    from ct_laboratory_b200.tomography.staticct_projector_3d import staticct_ray_tiling
    from ct_laboratory_b200.workloads import WORKLOADS
    w = WORKLOADS["static512"]
    p = w.projector(torch.device(DEV))
    x = w.phantom(device=DEV)
    per = p.src.shape[0] // w.n_view
    views = (0, 40, 80, 200)
    idx = torch.cat([torch.arange(v * per, (v + 1) * per, device=DEV) for v in views])
    src, dst = p.src[idx].contiguous(), p.dst[idx].contiguous()
    y = torch.rand(idx.numel(), device=DEV, generator=torch.Generator(device=DEV).manual_seed(2))
    Mi, b = torch.inverse(p.M).contiguous(), p.b
    rf = ref.forward_project_3d_on_the_fly_cuda(x, src, dst, Mi, b).cpu().numpy()
    rb = ref.back_project_3d_on_the_fly_cuda(y, src, dst, Mi, b, *w.n).cpu().numpy()
    til = staticct_ray_tiling(len(views) * w.modules_per_source, w.det_nx, w.det_ny, voxel_rule=p.ray_tiling.voxel_rule)
    assert til.tile_rows == 16
    for t in (til, None):
        f = _C.forward_project_3d_on_the_fly_cuda(x, src, dst, Mi, b, tiling=t)
        a = _C.back_project_3d_on_the_fly_cuda(y, src, dst, Mi, b, *w.n, tiling=t)
        assert rel_err(f.cpu().numpy(), rf) < 1e-5
        assert rel_err(a.cpu().numpy(), rb) < 1e-5
    # the reproducible (fixed-point) adjoint, 16-lane column walk
    from ct_laboratory_b200.tomography import back_project_3d_fixed_cuda
    fx = back_project_3d_fixed_cuda(y, src, dst, p.M, b, *w.n, tiling=til, M_inv=Mi)
    assert rel_err(fx.cpu().numpy(), rb.reshape(fx.shape)) < 1e-5
