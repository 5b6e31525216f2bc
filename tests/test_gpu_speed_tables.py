"""Speed and parity of the intersection-table paths (float and uint16
compressed) against the reference's own CUDA kernels, on a StaticCT ring the
size of the reference's published benchmark scan (workload static512: 240
views, 2,949,120 rays, 512^2 x 64 voxels over 400 mm x 60 mm).

Every projector timing the reference publishes is for its uint16 tables on
its calibrated StaticCT ring (for instance 46.2 / 36.1 ms forward / adjoint at
512^2 x 64 on an H100, benchmark/README.md:102); that geometry file is not
available, so the ring here is a uniform one with the same ray count and
grid.

* Ours, on the whole scan: the float table (compute_intersections_3d), its
  uint16 compression with the reference CUDA encoder, forward / adjoint from
  the compressed and from the float table, and the on-the-fly walk for
  comparison: both voxel rules flat, and the crossing rule with the modules'
  16 rows per column tiled for the column walk (forward bitwise equal to
  the flat walk's).
* The reference's kernels (compiled from its sources into oracle/_ref), on
  every tenth view: table, compression, forward / adjoint from both tables.
  A ray's cost does not depend on the other rays, so rays per second on the
  sample stand for the scan.

Parity on the sampled rays: the reference's uint16 stream against ours
(fraction of differing entries reported, must be tiny), and forward /
adjoint from the reference's compressed table against ours within the
projector tolerance 1e-5.  Set CTLAB_PERF_OUT=<file> to have the figures
written as JSON.
"""
import json
import os

import numpy as np
import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu
DEV = "cuda"
TOL = 1e-5
SAMPLE_EVERY = 10  # views


@pytest.fixture(scope="module")
def ref():
    from oracle.build_ref import load_ref
    mod = load_ref()
    if mod is None:
        pytest.skip("reference CUDA build not present (python oracle/build_ref.py)")
    return mod


def _ms(fn, reps=5, flush=None):
    fn()
    torch.cuda.synchronize()
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


def _once_ms(fn):
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    out = fn()
    e1.record()
    torch.cuda.synchronize()
    return out, e0.elapsed_time(e1)


def test_static512_table_paths_vs_reference(ref):
    from ct_laboratory_b200 import _C
    from ct_laboratory_b200 import _native as N
    from ct_laboratory_b200.tomography import staticct_ray_tiling
    from ct_laboratory_b200.tomography._common import voxel_diag_len
    from ct_laboratory_b200.workloads import WORKLOADS
    w = WORKLOADS["static512"]
    p = w.projector(torch.device(DEV))
    nx, ny, nz = w.n
    src, dst, b = p.src, p.dst, p.b
    Mi = torch.inverse(p.M).contiguous()
    vdl = voxel_diag_len(p.M)
    n_ray = src.shape[0]
    assert n_ray == w.n_ray == 2_949_120
    x = w.phantom(device=DEV)
    y = torch.rand(n_ray, device=DEV, generator=torch.Generator(device=DEV).manual_seed(1))
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=DEV)
    res = {"workload": w.name, "n_ray": n_ray, "grid": list(w.n)}

    with torch.no_grad():
        # ---- ours, whole scan
        _C.compute_intersections_3d(nx, ny, nz, src[:4096], dst[:4096], Mi, b)  # warm-up
        tv, res["ours_table_ms"] = _once_ms(lambda: _C.compute_intersections_3d(nx, ny, nz, src, dst, Mi, b))
        (u16, st, sc), res["ours_compress_ms"] = _once_ms(lambda: _C.compress_tvals_3d_cuda(tv, src, dst, vdl))
        res["n_int"] = int(tv.shape[1])
        res["table_bytes"] = {"float": tv.numel() * 4, "uint16": u16.numel() * 2 + 8 * n_ray}
        res["ours_float_ms"] = [_ms(lambda: _C.forward_project_3d_cuda(x, tv, src, dst, Mi, b), flush=flush),
                                _ms(lambda: _C.back_project_3d_cuda(y, tv, src, dst, Mi, b, nx, ny, nz), flush=flush)]
        res["ours_compressed_ms"] = [
            _ms(lambda: _C.forward_project_3d_compressed_cuda(x, u16, st, sc, src, dst, Mi, b), flush=flush),
            _ms(lambda: _C.back_project_3d_compressed_cuda(y, u16, st, sc, src, dst, Mi, b, nx, ny, nz), flush=flush)]
        cross = N.flat_opts(voxel_rule=N.VOXEL_CROSSING, block_threads=128)
        col16 = staticct_ray_tiling(n_ray // (w.det_nx * w.det_ny), w.det_nx, w.det_ny, voxel_rule=N.VOXEL_CROSSING)
        assert torch.equal(_C.forward_project_3d_on_the_fly_cuda(x, src, dst, Mi, b, tiling=col16),
                           _C.forward_project_3d_on_the_fly_cuda(x, src, dst, Mi, b, tiling=cross))
        res["ours_on_the_fly_ms"] = {
            "midpoint": [_ms(lambda: _C.forward_project_3d_on_the_fly_cuda(x, src, dst, Mi, b), flush=flush),
                         _ms(lambda: _C.back_project_3d_on_the_fly_cuda(y, src, dst, Mi, b, nx, ny, nz),
                             flush=flush)],
            "crossing": [_ms(lambda: _C.forward_project_3d_on_the_fly_cuda(x, src, dst, Mi, b, tiling=cross),
                             flush=flush),
                         _ms(lambda: _C.back_project_3d_on_the_fly_cuda(y, src, dst, Mi, b, nx, ny, nz, tiling=cross),
                             flush=flush)],
            "crossing_column_walk": [
                _ms(lambda: _C.forward_project_3d_on_the_fly_cuda(x, src, dst, Mi, b, tiling=col16), flush=flush),
                _ms(lambda: _C.back_project_3d_on_the_fly_cuda(y, src, dst, Mi, b, nx, ny, nz, tiling=col16),
                    flush=flush)]}

        # ---- the sample of whole views
        per_view = w.modules_per_source * w.det_nx * w.det_ny
        n_view = n_ray // per_view
        idx = torch.cat([torch.arange(v * per_view, (v + 1) * per_view, device=DEV)
                         for v in range(0, n_view, SAMPLE_EVERY)])
        n_s = int(idx.numel())
        ss, ds, ys = src[idx].contiguous(), dst[idx].contiguous(), y[idx].contiguous()
        u16s, sts, scs = u16[idx].contiguous(), st[idx].contiguous(), sc[idx].contiguous()
        del tv
        ref.compute_intersections_3d(nx, ny, nz, ss[:4096], ds[:4096], Mi, b)  # warm-up
        tv_r, res["ref_table_ms_sample"] = _once_ms(lambda: ref.compute_intersections_3d(nx, ny, nz, ss, ds, Mi, b))
        (u16r, str_, scr), res["ref_compress_ms_sample"] = _once_ms(
            lambda: ref.compress_tvals_3d_cuda(tv_r, ss, ds, vdl))
        res["ref_float_ms_sample"] = [
            _ms(lambda: ref.forward_project_3d_cuda(x, tv_r, ss, ds, Mi, b), reps=3, flush=flush),
            _ms(lambda: ref.back_project_3d_cuda(ys, tv_r, ss, ds, Mi, b, nx, ny, nz), reps=3, flush=flush)]
        holder = {}
        res["ref_compressed_ms_sample"] = [
            _ms(lambda: holder.__setitem__("f", ref.forward_project_3d_compressed_cuda(x, u16r, str_, scr, ss, ds,
                                                                                      Mi, b)), reps=3, flush=flush),
            _ms(lambda: holder.__setitem__("b", ref.back_project_3d_compressed_cuda(ys, u16r, str_, scr, ss, ds, Mi, b,
                                                                                   nx, ny, nz)), reps=3, flush=flush)]

        # ---- parity on the sample
        res["uint16_mismatch_fraction"] = float((u16r != u16s).double().mean())
        res["start_scale_max_abs_diff"] = [float((str_ - sts).abs().max()), float((scr - scs).abs().max())]
        of = _C.forward_project_3d_compressed_cuda(x, u16s, sts, scs, ss, ds, Mi, b)
        ob = _C.back_project_3d_compressed_cuda(ys, u16s, sts, scs, ss, ds, Mi, b, nx, ny, nz)
        res["parity_compressed_rel"] = [rel_err(of.cpu().numpy(), holder["f"].cpu().numpy()),
                                        rel_err(ob.cpu().numpy(), holder["b"].cpu().numpy())]

    scale = n_ray / n_s
    ours_c = n_ray / (sum(res["ours_compressed_ms"]) / 1e3)
    ref_c = n_s / (sum(res["ref_compressed_ms_sample"]) / 1e3)
    res.update({"sample_rays": n_s, "sample_views_every": SAMPLE_EVERY,
                "ref_compressed_ms_full_extrapolated": [t * scale for t in res["ref_compressed_ms_sample"]],
                "ref_float_ms_full_extrapolated": [t * scale for t in res["ref_float_ms_sample"]],
                "ref_table_ms_full_extrapolated": res["ref_table_ms_sample"] * scale,
                "ours_compressed_grays_s": ours_c / 1e9, "ref_compressed_grays_s": ref_c / 1e9,
                "speedup_compressed": ours_c / ref_c,
                "speedup_table_build": res["ref_table_ms_sample"] * scale / res["ours_table_ms"]})
    print(json.dumps(res))
    out = os.environ.get("CTLAB_PERF_OUT")
    if out:
        with open(out, "w") as f:
            json.dump(res, f, indent=1)
    assert res["uint16_mismatch_fraction"] < 1e-4, res
    assert max(res["parity_compressed_rel"]) < TOL, res
    assert res["speedup_compressed"] >= 1.0, res
