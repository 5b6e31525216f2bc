"""The drop-in seen from the reference's side.

The reference's own Python projector layers (its ct_laboratory/tomography
package: modules, autograd Functions, function API, geometry classes, subset
wrappers, tables on disk), staged into oracle/_ref/py by
oracle/stage_ref_python.py, are imported twice: once with
``sys.modules["ct_laboratory._C"] = ct_laboratory_b200._C`` (the alias a
maintainer adds to switch) and once over the reference's own
compiled module (oracle/_ref, built by oracle/build_ref.py).  The same
seeded calls through both must agree within the projector tolerance 1e-5:
argument orders, M^-1 conventions, squeeze rules, table formats and the
reference's own quirks (its no-table adjoint inverts M twice,
ct_projector_3d_cuda.py:209-210, :319, and both _C modules receive what it
passes) all go through the reference's code unchanged.  Then this package's
classes read what the reference's classes wrote: a ``save_tvals`` file
(ct_projector_3d_module.py:190-216) and an ordered-subset cache directory
(ct_projector_3d_subsets.py:85-97).
"""
import contextlib
import importlib
import os
import sys

import numpy as np
import pytest
import torch

from conftest import ROOT, rel_err

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")
TOL = 1e-5
CONE = dict(n_x=24, n_y=20, n_z=16, n_view=6, det_nx=32, det_ny=24, sid=100.0, sdd=150.0, det_spacing=0.8,
            voxel_size=0.5)
FAN = dict(n_row=32, n_col=28, n_view=10, n_det=40, sid=100.0, sdd=150.0, det_spacing=1.0, pixel_size=0.8)


@pytest.fixture(scope="module")
def modules():
    from oracle.build_ref import load_ref
    from oracle.stage_ref_python import staged_path
    ref_c = load_ref()
    staged = staged_path()
    if ref_c is None or staged is None:
        pytest.skip("reference build or staged layers missing (python __graft_entry__.py)")
    from ct_laboratory_b200 import _C as ours
    return staged, ours, ref_c


@contextlib.contextmanager
def reference_layers(staged, c_module):
    """The staged reference tomography package, freshly imported over c_module."""
    mine = lambda k: k == "ct_laboratory" or k.startswith("ct_laboratory.")  # noqa: E731
    saved = {k: sys.modules.pop(k) for k in [k for k in sys.modules if mine(k)]}
    sys.modules["ct_laboratory._C"] = c_module
    sys.path.insert(0, staged)
    try:
        yield importlib.import_module("ct_laboratory.tomography")
    finally:
        for k in [k for k in sys.modules if mine(k)]:
            del sys.modules[k]
        sys.path.remove(staged)
        sys.modules.update(saved)


def rnd(shape, seed):
    return torch.rand(shape, generator=torch.Generator(device=DEV).manual_seed(seed), device=DEV)


def run_reference_layers(tomo, workdir):
    """Seeded calls through the reference's classes and functions; returns
    numpy results keyed by name (and leaves its table files in workdir)."""
    os.makedirs(workdir, exist_ok=True)  # (the reference's save_tvals expects the directory)
    out = {}
    cone = tomo.ConeBeam3DProjector(**CONE, backend="cuda", device=DEV)
    n = (CONE["n_x"], CONE["n_y"], CONE["n_z"])
    x, y = rnd(n, 1), rnd(cone.src.shape[0], 2)
    out["cone_forward"] = cone(x)
    out["cone_back_project"] = cone.back_project(y)
    xg = x.clone().requires_grad_(True)
    (cone(xg) * y).sum().backward()
    out["cone_autograd_grad"] = xg.grad
    out["fn_forward_3d"] = tomo.forward_project_3d_cuda(x, None, cone.src, cone.dst, cone.M, cone.b)
    out["fn_back_3d"] = tomo.back_project_3d_cuda(y, None, cone.src, cone.dst, cone.M, cone.b, *n)
    table = tomo.CTProjector3DModule(*n, cone.M, cone.b, cone.src, cone.dst, backend="cuda", device=DEV,
                                     precomputed_intersections=True)
    out["table_forward"] = table(x)
    out["table_back_project"] = table.back_project(y)
    table.save_tvals(os.path.join(workdir, "ref_tvals.pt"))
    osp = tomo.OrderedSubsetProjector(cone, max_subset_size=1000, cache_dir=os.path.join(workdir, "cache"))
    out["subsets_forward"] = osp(x)
    out["subsets_back_project"] = osp.back_project(y)
    fan = tomo.FanBeam2DProjector(**FAN, backend="cuda", device=DEV)
    img, yf = rnd((FAN["n_row"], FAN["n_col"]), 3), rnd(fan.src.shape[0], 4)
    out["fan_forward"] = fan(img)
    out["fan_back_project"] = fan.back_project(yf)
    return {k: v.detach().float().cpu().numpy() for k, v in out.items()}, (x, y)


def test_reference_layers_over_our_C_match_its_own_C(modules, tmp_path):
    staged, ours, ref_c = modules
    with reference_layers(staged, ours) as tomo:
        assert tomo.ct_projector_3d_cuda._C is ours
        got, _ = run_reference_layers(tomo, str(tmp_path / "ours"))
    with reference_layers(staged, ref_c) as tomo:
        want, _ = run_reference_layers(tomo, str(tmp_path / "theirs"))
    assert sorted(got) == sorted(want)
    bad = {k: rel_err(got[k], want[k]) for k in got if not (got[k].shape == want[k].shape and
                                                             rel_err(got[k], want[k]) < TOL)}
    assert not bad, bad


def test_our_classes_read_the_reference_classes_files(modules, tmp_path):
    """A save_tvals file and a subset cache directory written by the
    reference's classes (over its own compiled module), read by ours."""
    from ct_laboratory_b200 import ConeBeam3DProjector, CTProjector3DModule, OrderedSubsetProjector
    staged, _, ref_c = modules
    work = str(tmp_path)
    with reference_layers(staged, ref_c) as tomo:
        want, (x, y) = run_reference_layers(tomo, work)
    cone = ConeBeam3DProjector(**CONE, device=DEV)
    n = (CONE["n_x"], CONE["n_y"], CONE["n_z"])
    mod = CTProjector3DModule(*n, cone.M, cone.b, cone.src, cone.dst, device=DEV)
    mod.load_tvals(os.path.join(work, "ref_tvals.pt"))
    assert mod.tvals_uint16 is not None and mod.precomputed_intersections
    assert rel_err(mod(x).cpu().numpy(), want["table_forward"]) < TOL
    assert rel_err(mod.back_project(y).cpu().numpy(), want["table_back_project"]) < TOL
    cache = os.path.join(work, "cache")
    files = sorted(os.listdir(cache))
    osp = OrderedSubsetProjector(cone, max_subset_size=1000, cache_dir=cache)
    assert osp.n_subsets == len(files) and osp.use_tables
    with torch.no_grad():
        assert rel_err(osp(x).cpu().numpy(), want["subsets_forward"]) < TOL
        assert rel_err(osp.back_project(y).cpu().numpy(), want["subsets_back_project"]) < TOL
    assert sorted(os.listdir(cache)) == files  # read, none rewritten or added
    np.testing.assert_equal(len(files), int(np.ceil(cone.src.shape[0] / 1000)))
