"""The batched projector's entry point for callers that cannot allocate GPU
memory (a plugin whose host application owns the device's memory, a
real-time loop that must not allocate mid-scan).

ctlab_project_batched_noalloc runs the batched forward / adjoint with its
work counter and scan table in a fixed array inside the library instead of
a caller-allocated workspace.  Checked here through the C ABI against the
planned entry points (ctlab_forward_project_batched /
ctlab_back_project_batched, via ScanBatch) on two calls in a row, with new
inputs and poisoned outputs between the calls so that a stale table or an
uncleared work counter would show.  Tolerance: the projector's 1e-5
(forward results are expected bitwise equal; adjoints differ only in the
order of float atomic additions).

This file sorts last so that a run stopping at the first failure has run
every other test first; it builds its own inputs and passes alone too.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = "cuda"
TOL = 1e-5


def _rel(a, b):
    a, b = a.double().cpu(), b.double().cpu()
    den = float(b.abs().max()) if b.numel() else 1.0
    return float((a - b).abs().max()) / max(den, 1e-30) if b.numel() else 0.0


def _projectors_2d():
    from ct_laboratory_b200 import FanBeam2DProjector
    rng = np.random.default_rng(11)
    return [FanBeam2DProjector(int(s), int(s), n_view=int(rng.integers(8, 24)), n_det=int(rng.integers(40, 80)),
                               sid=200.0, sdd=300.0, det_spacing=1.0, pixel_size=64.0 / int(s),
                               device=torch.device(DEV)) for s in rng.choice([24, 32, 48], size=5)]


def _projectors_3d():
    from ct_laboratory_b200 import ConeBeam3DProjector
    return [ConeBeam3DProjector(*n, n_view=v, det_nx=d[0], det_ny=d[1], sid=100.0, sdd=150.0, det_spacing=0.8,
                                voxel_size=0.5, voxel_rule=1, device=torch.device(DEV))
            for n, v, d in (((24, 20, 16), 7, (32, 32)), ((16, 16, 16), 5, (24, 64)), ((20, 24, 12), 6, (36, 32)))]


def _noalloc_scans(batch, img_out, sino_out):
    """The batch's scans in the batch's own order and layout, with the
    outputs redirected to separate buffers."""
    from ct_laboratory_b200 import _native as N
    kind, bt = batch.config["kind"], batch.config["block_threads"]
    scans = []
    for i in batch.order:
        s = batch._scan(i, kind, bt)
        s.sino_out, s.image_out = sino_out[i].data_ptr(), img_out[i].data_ptr()
        scans.append(s)
    return (N.Scan * len(scans))(*scans)


@pytest.mark.parametrize("make", [_projectors_2d, _projectors_3d])
def test_noalloc_entry_matches_planned_entry_twice(make):
    from ct_laboratory_b200 import _native as N
    from ct_laboratory_b200.batched import ScanBatch
    batch = ScanBatch(make())
    img_out = [torch.empty_like(t) for t in batch.images_out]
    sino_out = [torch.empty_like(t) for t in batch.sinos_out]
    arr = _noalloc_scans(batch, img_out, sino_out)
    n, bt, ctas = len(arr), batch.config["block_threads"], batch.config["n_cta"]
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    gen = torch.Generator(device=DEV)
    for call in range(2):
        gen.manual_seed(100 + call)  # new inputs on every call
        for t in batch.images_in + batch.sinos_in:
            t.copy_(torch.rand(t.shape, generator=gen, device=DEV))
        for t in img_out + sino_out:
            t.fill_(float("nan"))  # a call that skipped work would leave NaN
        batch.forward()
        batch.back()
        assert N.lib.ctlab_project_batched_noalloc(arr, n, 0, 0, bt, ctas, stream) == 0, N.lib.ctlab_last_error()
        assert N.lib.ctlab_project_batched_noalloc(arr, n, 1, 0, bt, ctas, stream) == 0, N.lib.ctlab_last_error()
        torch.cuda.synchronize()
        for i in range(n):
            assert not torch.isnan(sino_out[i]).any() and not torch.isnan(img_out[i]).any()
            assert _rel(sino_out[i], batch.sinos_out[i]) <= TOL, (call, i)
            assert _rel(img_out[i], batch.images_out[i]) <= TOL, (call, i)


def test_noalloc_entry_rejects_more_scans_than_its_scratch_holds():
    from ct_laboratory_b200 import _native as N
    from ct_laboratory_b200.batched import ScanBatch
    batch = ScanBatch(_projectors_2d()[:1])
    one = _noalloc_scans(batch, batch.images_out, batch.sinos_out)[0]
    arr = (N.Scan * 65)(*([one] * 65))
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = N.lib.ctlab_project_batched_noalloc(arr, 65, 0, 0, 256, 0, stream)
    assert rc == 1 and b"at most 64 scans" in N.lib.ctlab_last_error()



def test_noalloc_entry_at_its_limit_of_64_scans():
    """64 scans (the most the fixed array holds), each with its own inputs
    and NaN-filled outputs, against the planned batch of the same 64 scans:
    a bad table entry or a work counter that stopped early would leave one
    of them wrong or NaN."""
    from ct_laboratory_b200 import _native as N
    from ct_laboratory_b200.batched import ScanBatch
    p = _projectors_2d()[0]
    batch = ScanBatch([p] * 64)
    img_out = [torch.empty_like(t) for t in batch.images_out]
    sino_out = [torch.empty_like(t) for t in batch.sinos_out]
    arr = _noalloc_scans(batch, img_out, sino_out)
    assert len(arr) == 64
    gen = torch.Generator(device=DEV).manual_seed(7)
    for t in batch.images_in + batch.sinos_in:
        t.copy_(torch.rand(t.shape, generator=gen, device=DEV))
    for t in img_out + sino_out:
        t.fill_(float("nan"))
    batch.forward()
    batch.back()
    bt, ctas = batch.config["block_threads"], batch.config["n_cta"]
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for adjoint in (0, 1):
        assert N.lib.ctlab_project_batched_noalloc(arr, 64, adjoint, 0, bt, ctas, stream) == 0, \
            N.lib.ctlab_last_error()
    torch.cuda.synchronize()
    for i in range(64):
        assert not torch.isnan(sino_out[i]).any() and not torch.isnan(img_out[i]).any(), i
        assert _rel(sino_out[i], batch.sinos_out[i]) <= TOL, i
        assert _rel(img_out[i], batch.images_out[i]) <= TOL, i
