"""Subset and multi-rotation projectors on the GPU kernels (the reference's
tomography/ct_projector_3d_subsets.py and ct_projector_3d_multirot.py).

Ordered subsets against the core module (with and without tables, tables
from the core, from a cache directory written under the reference's file
names); random subsets against the core restricted to the same rays;
multi-rotation windows through one batched launch against the reference's
per-rotation loop, the adjoint identity and autograd.  Tolerance 1e-5 (the
projector's); forward results of the same kernel on the same rays are
expected bitwise equal."""
import os

import numpy as np
import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")
TOL = 1e-5


def cone(**kw):
    from ct_laboratory_b200 import ConeBeam3DProjector
    args = dict(n_x=24, n_y=20, n_z=16, n_view=10, det_nx=32, det_ny=24, sid=100.0, sdd=150.0, det_spacing=0.8,
                voxel_size=0.5, device=DEV)
    args.update(kw)
    return ConeBeam3DProjector(**args)


def rnd(*shape, seed=0):
    return torch.rand(*shape, generator=torch.Generator(device=DEV).manual_seed(seed), device=DEV)


def test_ordered_subsets_without_tables_is_the_core_projector():
    from ct_laboratory_b200 import OrderedSubsetProjector
    core = cone()
    osp = OrderedSubsetProjector(core, max_subset_size=1000)
    assert osp.n_subsets == int(np.ceil(core.src.shape[0] / 1000)) and not osp.use_tables
    x, y = rnd(24, 20, 16), rnd(core.src.shape[0], seed=1)
    assert torch.equal(osp(x), core(x))
    assert rel_err(osp.back_project(y).cpu().numpy(), core.back_project(y).cpu().numpy()) < TOL


def test_ordered_subsets_with_core_tables_match_whole_table_projection():
    from ct_laboratory_b200 import CTProjector3DModule, OrderedSubsetProjector
    base = cone()
    core = CTProjector3DModule(24, 20, 16, base.M, base.b, base.src, base.dst, device=DEV,
                               precomputed_intersections=True)
    osp = OrderedSubsetProjector(core, max_subset_size=997)
    assert osp.use_tables and osp.n_subsets > 1
    x, y = rnd(24, 20, 16), rnd(core.src.shape[0], seed=2)
    assert torch.equal(osp(x), core(x))
    assert rel_err(osp.back_project(y).cpu().numpy(), core.back_project(y).cpu().numpy()) < TOL
    xb = rnd(2, 24, 20, 16, seed=3)  # batched volumes
    assert torch.equal(osp(xb), core(xb))


def test_ordered_subsets_cache_dir_files_and_reload(tmp_path):
    from ct_laboratory_b200 import CTProjector3DModule, OrderedSubsetProjector
    core = cone()
    osp = OrderedSubsetProjector(core, max_subset_size=1500, cache_dir=str(tmp_path))
    x = rnd(24, 20, 16, seed=4)
    first = osp(x)
    names = sorted(os.listdir(tmp_path))
    b = osp.subset_boundaries
    want = sorted(f"tvals_subset{j:04d}_rays{int(b[j])}-{int(b[j + 1])}_nx24_ny20_nz16.pt"
                  for j in range(osp.n_subsets))
    assert names == want
    again = OrderedSubsetProjector(core, max_subset_size=1500, cache_dir=str(tmp_path))(x)
    assert torch.equal(first, again)
    # the cached tables are precompute_tvals_stitched's (the reference's CUDA
    # uint16 encoder, with its clamping): the same as one whole-scan module
    # holding the stitched tables of all rays
    from ct_laboratory_b200 import precompute_tvals_stitched
    tabs = precompute_tvals_stitched(24, 20, 16, core.M, core.b, core.src, core.dst, verbose=False)
    whole = CTProjector3DModule(24, 20, 16, core.M, core.b, core.src, core.dst, device=DEV, tvals=tabs)
    assert torch.equal(first, whole(x))


def test_random_subset_is_the_core_on_those_rays():
    from ct_laboratory_b200 import RandomSubsetProjector
    core = cone()
    rsp = RandomSubsetProjector(core, subset_size=500, seed=7)
    torch.manual_seed(7)
    idx = torch.randperm(core.src.shape[0])[:500]
    assert torch.equal(rsp.current_indices, idx)
    x = rnd(24, 20, 16, seed=5)
    # the subset has no detector layout (flat launch, per-lane walk) while the
    # core takes the column walk: the same segments and voxels, summed in
    # another order
    assert rel_err(rsp(x).cpu().numpy(), core(x)[idx.to(DEV)].cpu().numpy()) < TOL
    rsp.randomize_projector(seed=8)
    assert not torch.equal(rsp.current_indices, idx)


@pytest.mark.parametrize("mode", ["repeat", "reflect", "zeros"])
def test_multirotation_batched_matches_per_rotation_loop(mode):
    from ct_laboratory_b200 import MultiRotationProjector
    base = cone(n_z=12)
    mr = MultiRotationProjector(base, n_rotations=5, shift_offset=6.0, n_z_window=12, padding_mode=mode,
                                reflection_padding_slices=3 if mode == "reflect" else None)
    x = rnd(24, 20, 30, seed=6)
    sino = mr(x)
    assert sino.shape == (base.src.shape[0], 5)
    loop = torch.stack([base(mr._extract_volume_slice(x, *mr._get_rotation_z_bounds(30, i))) for i in range(5)],
                       dim=1)
    assert torch.equal(sino, loop)
    y = rnd(base.src.shape[0], 5, seed=7)
    bp = mr.back_project(y, 30)
    assert bp.shape == (24, 20, 30)
    lhs, rhs = float((sino.double() * y.double()).sum()), float((x.double() * bp.double()).sum())
    assert abs(lhs - rhs) < 1e-5 * abs(lhs)


def test_multirotation_autograd_and_subset_base():
    from ct_laboratory_b200 import CTProjector3DModule, MultiRotationProjector, OrderedSubsetProjector
    base = cone(n_z=12)
    mr = MultiRotationProjector(base, n_rotations=3, shift_offset=8.0, n_z_window=12, padding_mode="zeros")
    x = rnd(24, 20, 28, seed=8).requires_grad_(True)
    w = rnd(base.src.shape[0], 3, seed=9)
    (mr(x) * w).sum().backward()
    assert rel_err(x.grad.cpu().numpy(), mr.back_project(w, 28).cpu().numpy()) < TOL
    # ordered subsets with tables under the rotations: tables once per subset
    tab = CTProjector3DModule(24, 20, 12, base.M, base.b, base.src, base.dst, device=DEV,
                              precomputed_intersections=True)
    mr_s = MultiRotationProjector(OrderedSubsetProjector(tab, max_subset_size=1200), n_rotations=3,
                                  shift_offset=8.0, n_z_window=12, padding_mode="zeros")
    mr_t = MultiRotationProjector(tab, n_rotations=3, shift_offset=8.0, n_z_window=12, padding_mode="zeros")
    with torch.no_grad():
        assert torch.equal(mr_s(x), mr_t(x))
        assert rel_err(mr_s.back_project(w, 28).cpu().numpy(), mr_t.back_project(w, 28).cpu().numpy()) < TOL
