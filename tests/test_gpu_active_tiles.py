"""Active-tile launches (ctlab_active_tiles + the *_tiles entry points).

The tiles listed are those holding a ray the walks charge; launching only
them must give the full launch's results: the forward bitwise (the same
walks, and 0 for every ray of a skipped tile), the adjoint to the order of
its float additions (1e-6 of the maximum), and the reproducible adjoint
bitwise.  The geometry has a detector much wider and taller than the
volume's shadow, so most tiles are skipped; the cases cover both voxel
rules, 32- and 16-row tiles, batches of volumes, and an empty list.
"""
import numpy as np
import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu
DEV = "cuda"


def cone(rows=32, rule=0, det=(96, 80), n=(24, 20, 16)):
    from ct_laboratory_b200 import ConeBeam3DProjector
    return ConeBeam3DProjector(*n, n_view=9, det_nx=det[0], det_ny=det[1], sid=100.0, sdd=150.0, det_spacing=0.8,
                               voxel_size=0.5, device=torch.device(DEV), tile_rows=rows, voxel_rule=rule)


@pytest.mark.parametrize("rows,rule", [(32, 0), (32, 1), (16, 0), (16, 1)])
def test_tile_list_launches_equal_full_launches(rows, rule):
    from ct_laboratory_b200 import _C
    from ct_laboratory_b200 import _native as N
    p = cone(rows, rule)
    act = p._launch_tiling()
    n_all = int(N.lib.ctlab_tile_count(p.src.shape[0], N.tiling_ref(p.ray_tiling)))
    n_act = act.active[1]
    assert 0 < n_act < n_all // 2, (n_act, n_all)  # most of the detector misses the volume
    tiles = act.active[0].cpu().numpy()
    assert np.all(np.diff(tiles) > 0) and tiles[0] >= 0 and tiles[-1] < n_all  # ascending, in range
    g = torch.Generator(device=DEV).manual_seed(rows + rule)
    for batch in (1, 3):
        x = torch.rand(batch, p.n_x, p.n_y, p.n_z, generator=g, device=DEV)
        y = torch.rand(batch, p.src.shape[0], generator=g, device=DEV)
        args = (p.src, p.dst, p.M_inv, p.b)
        f_full = _C.forward_project_3d_on_the_fly_cuda(x, *args, tiling=p.ray_tiling)
        f_act = _C.forward_project_3d_on_the_fly_cuda(x, *args, tiling=act)
        assert torch.equal(f_full, f_act)
        b_full = _C.back_project_3d_on_the_fly_cuda(y, *args, p.n_x, p.n_y, p.n_z, tiling=p.ray_tiling)
        b_act = _C.back_project_3d_on_the_fly_cuda(y, *args, p.n_x, p.n_y, p.n_z, tiling=act)
        assert rel_err(b_act.cpu().numpy(), b_full.cpu().numpy()) < 1e-6
    # the module's own calls take the list
    with torch.no_grad():
        assert torch.equal(p.forward_project(x[0]), f_full[0])


def test_tile_lists_follow_the_geometry_and_the_empty_list():
    from ct_laboratory_b200 import _C
    from ct_laboratory_b200 import _native as N
    p = cone()
    a1 = p._launch_tiling()
    assert p._launch_tiling() is a1  # cached
    with torch.no_grad():
        p.dst[:, 2] += 1000.0  # every ray now passes far above the volume
    a2 = p._launch_tiling()
    assert a2 is not a1 and a2.active[1] == 0
    x = torch.rand(p.n_x, p.n_y, p.n_z, device=DEV)
    out = _C.forward_project_3d_on_the_fly_cuda(x, p.src, p.dst, p.M_inv, p.b, tiling=a2)
    assert int(torch.count_nonzero(out)) == 0
    full = _C.forward_project_3d_on_the_fly_cuda(x, p.src, p.dst, p.M_inv, p.b, tiling=p.ray_tiling)
    assert int(torch.count_nonzero(full)) == 0
    # a list longer than the tiling is refused on the host
    n_all = int(N.lib.ctlab_tile_count(p.src.shape[0], N.tiling_ref(p.ray_tiling)))
    bogus = torch.zeros(n_all + 1, dtype=torch.int32, device=DEV)
    o = torch.empty(1, p.src.shape[0], device=DEV)
    rc = N.lib.ctlab_forward_project_3d_on_the_fly_tiles(N.ptr(x), 1, p.n_x, p.n_y, p.n_z, N.ptr(p.src),
                                                         N.ptr(p.dst), p.src.shape[0], N.ptr(p.M_inv), N.ptr(p.b),
                                                         N.ptr(o), N.tiling_ref(p.ray_tiling), N.ptr(bogus),
                                                         n_all + 1, N.stream_of(x))
    assert rc != 0


def test_reproducible_adjoint_with_a_tile_list_is_bitwise_the_same():
    """The fixed-point adjoint walking only the listed tiles gives the full
    launch's bits (integer sums of the same contributions)."""
    from ct_laboratory_b200.tomography import back_project_3d_fixed_cuda
    p = cone()
    act = p._launch_tiling()
    y = torch.rand(p.src.shape[0], device=DEV)
    a = back_project_3d_fixed_cuda(y, p.src, p.dst, p.M, p.b, p.n_x, p.n_y, p.n_z, tiling=p.ray_tiling,
                                   M_inv=p.M_inv)
    b = back_project_3d_fixed_cuda(y, p.src, p.dst, p.M, p.b, p.n_x, p.n_y, p.n_z, tiling=act, M_inv=p.M_inv)
    assert torch.equal(a, b)


def test_bare_C_calls_list_their_tiles_and_follow_new_values():
    """_C calls without a launch hint (the reference's wrappers) launch the
    detected layout's active tiles: results equal the full launch's, a fresh
    M^-1 tensor with the same values reuses the list, and new values of b
    (the volume moved) give a new list and the full launch's results again."""
    from ct_laboratory_b200 import _C
    from ct_laboratory_b200 import _layout
    p = cone(det=(96, 64))  # (the layout detection takes row counts that are multiples of 32)
    x = torch.rand(1, p.n_x, p.n_y, p.n_z, device=DEV)
    y = torch.rand(1, p.src.shape[0], device=DEV)
    full_t = _layout.detect_tiling(p.src, p.dst)
    assert full_t is not None and full_t.n_view > 0
    _C._BARE_TILES.clear()
    for b in (p.b, p.b + torch.tensor([0.0, 0.0, 3.0], device=DEV)):
        b = b.contiguous()
        Mi = torch.inverse(p.M).contiguous()
        f = _C.forward_project_3d_on_the_fly_cuda(x, p.src, p.dst, Mi, b)
        a = _C.back_project_3d_on_the_fly_cuda(y, p.src, p.dst, Mi, b, p.n_x, p.n_y, p.n_z)
        f_full = _C.forward_project_3d_on_the_fly_cuda(x, p.src, p.dst, Mi, b, tiling=full_t)
        a_full = _C.back_project_3d_on_the_fly_cuda(y, p.src, p.dst, Mi, b, p.n_x, p.n_y, p.n_z, tiling=full_t)
        assert torch.equal(f, f_full)
        assert rel_err(a.cpu().numpy(), a_full.cpu().numpy()) < 1e-6
        opts = next(reversed(_C._BARE_TILES.values()))[4]
        assert opts.active is not None and opts.active[1] > 0
        # a fresh M^-1 with the same values: the same list
        n_entries = len(_C._BARE_TILES)
        _C.forward_project_3d_on_the_fly_cuda(x, p.src, p.dst, torch.inverse(p.M).contiguous(), b)
        assert len(_C._BARE_TILES) == n_entries and next(reversed(_C._BARE_TILES.values()))[4] is opts
    assert len(_C._BARE_TILES) == 1  # new values replaced the entry (same key, new contents)
