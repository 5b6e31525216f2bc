"""Many scans in one persistent launch (ScanBatch over ctlab_batch_plan /
ctlab_{forward,back}_project_batched), checked against the per-scan loop of
the same kernels, the reference's golden outputs, CUDA-graph replay and the
autotuner.

Forward results are bitwise those of the single-scan entry points (same walk,
same order of additions); adjoints agree up to the order of the float
atomic additions, checked at the projector tolerance 1e-5.  Against the
torch-path goldens the tolerance is TOL_TORCH = 5e-5 (the spread between the
reference's own torch and CUDA paths; see test_gpu_parity.py).
"""
import math

import numpy as np
import pytest
import torch

from conftest import load_golden, rel_err

pytestmark = pytest.mark.gpu
DEV = "cuda"
TOL = 1e-5
TOL_TORCH = 5e-5


def _rot2(theta):
    c, s = math.cos(theta), math.sin(theta)
    return torch.tensor([[c, -s], [s, c]], dtype=torch.float32)


def uneven_2d(seed=0, n=10):
    """Fan-beam and StaticCT-ring scans of uneven image size, view count and
    detector size (small versions of the batched-scan workload)."""
    from ct_laboratory_b200 import FanBeam2DProjector, UniformStaticCTProjector2D, standard_image_transform_2d
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        side = int(rng.choice([24, 32, 48, 64]))
        pixel = 64.0 / side
        if i % 2 == 0:
            out.append(FanBeam2DProjector(side, side, n_view=int(rng.integers(6, 30)), n_det=int(rng.integers(40, 96)),
                                          sid=200.0, sdd=300.0, det_spacing=1.0, pixel_size=pixel,
                                          device=torch.device(DEV)))
        else:
            n_source, n_frame = int(rng.integers(4, 12)), 2
            M, b = standard_image_transform_2d(side, side, pixel, pixel)
            Mg = torch.stack([_rot2(0.1 * f) for f in range(n_frame)])
            bg = torch.zeros(n_frame, 2)
            act = torch.ones(n_frame, n_source, dtype=torch.bool)
            out.append(UniformStaticCTProjector2D(side, side, M, b, n_source, 90.0, 8, 85.0, 16, 1.0, Mg, bg, act,
                                                  device=torch.device(DEV)))
    return out


def uneven_3d(seed=0):
    from ct_laboratory_b200 import ConeBeam3DProjector
    rng = np.random.default_rng(seed)
    out = []
    for n, views, det in (((24, 20, 16), 9, (32, 24)), ((32, 28, 24), 12, (40, 32)), ((16, 16, 16), 6, (24, 64)),
                          ((20, 24, 12), 7, (36, 40))):
        out.append(ConeBeam3DProjector(*n, n_view=views, det_nx=det[0], det_ny=det[1], sid=100.0, sdd=150.0,
                                       det_spacing=0.8, voxel_size=float(rng.choice([0.5, 1.0])), voxel_rule=1,
                                       device=torch.device(DEV)))
    return out


def _fill(batch, seed=1):
    g = torch.Generator(device=DEV).manual_seed(seed)
    for t in (batch.images_in or []) + (batch.sinos_in or []):
        t.copy_(torch.rand(t.shape, generator=g, device=DEV))


def _snap(ts):
    return [t.clone() for t in ts]


def _check_against_loop(batch):
    batch.forward()
    batch.back()
    f, b = _snap(batch.sinos_out), _snap(batch.images_out)
    batch.forward_loop()
    batch.back_loop()
    torch.cuda.synchronize()
    for i in range(len(f)):
        assert torch.equal(f[i], batch.sinos_out[i]), f"scan {i}: batched forward differs from the per-scan loop"
        assert rel_err(b[i].cpu().numpy(), batch.images_out[i].cpu().numpy()) < TOL, f"scan {i} adjoint"


@pytest.mark.parametrize("block_threads", [128, 256])
@pytest.mark.parametrize("kind", ["flat", "grid32", "grid64", "vgrid32", "vgrid64"])
def test_batched_2d_equals_per_scan_loop(kind, block_threads):
    from ct_laboratory_b200.batched import ScanBatch
    batch = ScanBatch(uneven_2d(), block_threads=block_threads, kind=kind)
    _fill(batch)
    _check_against_loop(batch)


@pytest.mark.parametrize("kind", ["flat", "col32", "col64"])
def test_batched_3d_equals_per_scan_loop(kind):
    from ct_laboratory_b200.batched import ScanBatch
    batch = ScanBatch(uneven_3d(), kind=kind)
    assert batch.config["mode"] == "loop" and batch.config_adj["mode"] == "persistent"  # the 3-D defaults
    _fill(batch)
    _check_against_loop(batch)
    batch.configure(kind=kind, mode="persistent")  # and the persistent forward
    _check_against_loop(batch)


def uneven_static_3d():
    """StaticCT rings (16 rows per module column, crossing rule: col16 tiles)
    of uneven grid, source count and module width."""
    from ct_laboratory_b200.tomography import UniformStaticCTProjector3D, standard_image_transform_3d
    out = []
    for n, n_source, n_cols, n_frame in (((32, 28, 12), 5, 8, 2), ((24, 24, 16), 7, 4, 1), ((20, 30, 10), 4, 6, 3)):
        M, b = standard_image_transform_3d(*n, 1.0, 1.0, 0.5)
        Mg = torch.stack([_rot3(0.2 * f) for f in range(n_frame)])
        act = torch.ones(n_frame, n_source, dtype=torch.bool)
        out.append(UniformStaticCTProjector3D(*n, n_source, 60.0, 0.0, 12, 55.0, n_cols, 16, 3.0, 1.0, 0.0, Mg,
                                              torch.zeros(n_frame, 3), act, 4, M, b, device=torch.device(DEV),
                                              voxel_rule=1))
    return out


def _rot3(theta):
    c, s = math.cos(theta), math.sin(theta)
    return torch.tensor([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]], dtype=torch.float32)


@pytest.mark.parametrize("mode", ["auto", "persistent"])
def test_batched_static_rings_col16(mode):
    """16-row detector columns: the persistent adjoint's two-group column walk
    and both forward modes against the per-scan loop."""
    from ct_laboratory_b200.batched import ScanBatch, tile_kinds
    projs = uneven_static_3d()
    assert all("col16" in tile_kinds(p) for p in projs)
    batch = ScanBatch(projs, block_threads=128)
    assert batch.config_adj["kind"] == ["col16"] * 3 and batch.config_adj["mode"] == "persistent"
    if mode == "persistent":
        batch.configure(block_threads=128, mode="persistent")
    _fill(batch)
    _check_against_loop(batch)


def test_batched_midpoint_rule_matches_goldens():
    """The reference's golden cases as scans of one batch each (2-D, 3-D), with
    the reference's voxel rule."""
    from ct_laboratory_b200 import CTProjector2DModule, CTProjector3DModule
    from ct_laboratory_b200 import _native as N
    from ct_laboratory_b200.batched import ScanBatch
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a)).to(DEV, torch.float32)  # noqa: E731
    for names, ndim in ((["kat2d", "fan2d", "static2d"], 2), (["kat3d", "cone3d", "affine3d", "edge3d", "static3d"], 3)):
        gs = [load_golden(n) for n in names]
        projs = []
        for g in gs:
            d = [int(v) for v in g["dims"]]
            if ndim == 2:
                projs.append(CTProjector2DModule(*d, T(g["M"]), T(g["b"]), T(g["src"]), T(g["dst"])))
            else:
                projs.append(CTProjector3DModule(*d, T(g["M"]), T(g["b"]), T(g["src"]), T(g["dst"]),
                                                 device=torch.device(DEV)))
        batch = ScanBatch(projs, voxel_rule=N.VOXEL_MIDPOINT, kind="flat")
        for i, g in enumerate(gs):
            batch.images_in[i].copy_(T(g["img"] if ndim == 2 else g["vol"]))
            batch.sinos_in[i].copy_(T(g["y"]))
        batch.forward()
        batch.back()
        torch.cuda.synchronize()
        for i, g in enumerate(gs):
            assert rel_err(batch.sinos_out[i].cpu().numpy(), g["fwd"]) < TOL_TORCH, names[i]
            assert rel_err(batch.images_out[i].cpu().numpy(), g["back"]) < TOL_TORCH, names[i]


def test_graph_replay_matches_eager():
    from ct_laboratory_b200.batched import ScanBatch
    batch = ScanBatch(uneven_2d(seed=3))
    _fill(batch, seed=4)
    graph = batch.capture()
    graph.replay()
    torch.cuda.synchronize()
    f, b = _snap(batch.sinos_out), _snap(batch.images_out)
    # new inputs in place; the captured graph sees them
    _fill(batch, seed=5)
    graph.replay()
    torch.cuda.synchronize()
    f2, b2 = _snap(batch.sinos_out), _snap(batch.images_out)
    batch.forward()
    batch.back()
    torch.cuda.synchronize()
    for i in range(len(f)):
        assert not torch.equal(f[i], f2[i])
        assert torch.equal(f2[i], batch.sinos_out[i])
        assert rel_err(b2[i].cpu().numpy(), batch.images_out[i].cpu().numpy()) < TOL
    del graph


def test_autotuner_picks_a_measured_candidate():
    from ct_laboratory_b200.batched import Autotuner, ScanBatch
    batch = ScanBatch(uneven_2d(seed=6))
    tuner = Autotuner()
    cfg = batch.autotune(reps=2, tuner=tuner)
    trials = tuner.trials[batch.signature()]
    assert set(trials) == {"fwd", "adj"}
    for d in ("fwd", "adj"):  # 2 modes x 2 block sizes x 5 tile kinds, each direction timed on its own
        assert len(trials[d]) == 20 and trials[d] == sorted(trials[d])
    assert (cfg["block_threads"], cfg["kind"], cfg["mode"]) == trials["fwd"][0][1:]
    assert (batch.config_adj["block_threads"], batch.config_adj["kind"], batch.config_adj["mode"]) == \
        trials["adj"][0][1:]
    again = batch.autotune(tuner=tuner)  # cached: no new trials
    assert again["kind"] == cfg["kind"] and len(tuner.trials) == 1
    _fill(batch)
    _check_against_loop(batch)


def test_empty_scan_and_accumulate():
    from ct_laboratory_b200 import CTProjector2DModule
    from ct_laboratory_b200.batched import ScanBatch
    projs = uneven_2d(seed=7, n=3)
    empty = CTProjector2DModule(16, 16, torch.eye(2, device=DEV), torch.zeros(2, device=DEV),
                                torch.zeros(0, 2, device=DEV), torch.zeros(0, 2, device=DEV))
    batch = ScanBatch(projs + [empty])
    _fill(batch)
    batch.images_out[3].fill_(7.0)
    batch.forward()
    batch.back()
    torch.cuda.synchronize()
    assert float(batch.images_out[3].abs().max()) == 0.0  # zeroed, nothing added
    first = _snap(batch.images_out)
    batch.back(accumulate=True)
    torch.cuda.synchronize()
    for i in range(3):
        assert rel_err(batch.images_out[i].cpu().numpy(), (2 * first[i]).cpu().numpy()) < TOL


def test_mixed_dimensions_rejected():
    from ct_laboratory_b200.batched import ScanBatch
    with pytest.raises(ValueError):
        ScanBatch(uneven_2d(n=2) + uneven_3d()[:1])
