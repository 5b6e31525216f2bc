"""The column walk's decisions per warp, against the per-lane walk and the
oracle, on geometries built to exercise each branch:

* a volume affine rotated about z only: a detector column's rays still share
  their index-space x-y line, so every warp takes the column walk;
* a volume tilted about x: world z leaks into the index-space y, the rays of
  a column no longer share their x-y line and every warp falls back to the
  per-lane walk inside the same launch;
* a tall detector close to the source: its outer rows are steeper in z than
  the crossing rule's column walk admits (|v_z| > 0.75 |v_xy|), so under
  that rule those warps fall back while the central rows' warps walk the
  column, in one launch; the midpoint rule's column walk takes several z
  planes per cell and walks every warp of it.

Under the crossing rule the detector-row tiling (column walk where it
applies) gives the forward bitwise equal to the flat launch (per-lane walk
everywhere).  Under the midpoint rule the column walk needs a diagonal M^-1
(the rotated and tilted affines walk per lane, bitwise as well) and, where it
runs, sums the same segments in another order: equal to 1e-6.  Adjoints are
equal up to the order of the float atomic additions (1e-6 here), and both
walks agree with the oracle's plane-sort walk within the projector tolerance
1e-5 under the midpoint rule, where that oracle is the reference's own rule.
"""
import math

import numpy as np
import pytest
import torch

from conftest import rel_err
from oracle import oracle as O

pytestmark = pytest.mark.gpu
DEV = "cuda"
TOL = 1e-5


def _rot(axis, deg):
    c, s = math.cos(math.radians(deg)), math.sin(math.radians(deg))
    if axis == "z":
        return np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]], np.float64)
    return np.array([[1, 0, 0], [0, c, -s], [0, s, c]], np.float64)


def _case(kind, seed):
    from ct_laboratory_b200.tomography import build_conebeam_3d_geometry
    n = np.array([36, 32, 24])
    voxel = 0.5
    if kind == "steep":  # 64 rows of 2 mm at 60 mm from the source, a volume 80 mm tall
        n = np.array([36, 32, 160])
        n_view, det, sid, sdd, pitch = 12, (40, 64), 40.0, 60.0, 2.0
    else:
        n_view, det, sid, sdd, pitch = 12, (40, 64), 120.0, 180.0, 0.4
    src, dst = build_conebeam_3d_geometry(n_view, det[0], det[1], sid, sdd, pitch)
    R = _rot("z", 30.0) if kind == "rot_z" else (_rot("x", 10.0) if kind == "tilt_x" else np.eye(3))
    M = (R @ np.diag([voxel] * 3)).astype(np.float32)
    b = (-(M.astype(np.float64) @ ((n - 1) / 2.0))).astype(np.float32)
    rng = np.random.default_rng(seed)
    vol = rng.random(tuple(n)).astype(np.float32)
    y = rng.random(src.shape[0]).astype(np.float32)
    return dict(n=n, M=M, Minv=O.minv(M), b=b, src=src.numpy(), dst=dst.numpy(), vol=vol, y=y, n_view=n_view,
                det=det)


def T(a):
    return torch.as_tensor(np.ascontiguousarray(a)).to(DEV, torch.float32)


@pytest.mark.parametrize("rule", [0, 1])
@pytest.mark.parametrize("kind", ["rot_z", "tilt_x", "steep"])
def test_column_walk_branches_match_per_lane_walk(kind, rule):
    from ct_laboratory_b200 import _C
    from ct_laboratory_b200 import _native as N
    c = _case(kind, seed=3)
    n_view, (nu, nv) = c["n_view"], c["det"]
    col = N.tiling(n_view, nv, nu, nv * nu, nu, 1, tile_rows=32, voxel_rule=rule, walk=N.WALK_COLUMN)
    flat = N.flat_opts(voxel_rule=rule)
    args = (T(c["src"]), T(c["dst"]), T(c["Minv"]), T(c["b"]))
    f_col = _C.forward_project_3d_on_the_fly_cuda(T(c["vol"]), *args, tiling=col)
    f_flat = _C.forward_project_3d_on_the_fly_cuda(T(c["vol"]), *args, tiling=flat)
    if rule == 1 or kind != "steep":
        assert torch.equal(f_col, f_flat)
    else:  # the midpoint column walk: the same segments summed in another order
        assert rel_err(f_col.cpu().numpy(), f_flat.cpu().numpy()) < 1e-6
    dims = [int(v) for v in c["n"]]
    b_col = _C.back_project_3d_on_the_fly_cuda(T(c["y"]), *args, *dims, tiling=col)
    b_flat = _C.back_project_3d_on_the_fly_cuda(T(c["y"]), *args, *dims, tiling=flat)
    assert rel_err(b_col.cpu().numpy(), b_flat.cpu().numpy()) < 1e-6
    if rule == 0:  # the oracle's plane sort is the reference's midpoint rule
        ref = O.fwd_planesort(c["vol"], c["Minv"], c["b"], c["src"], c["dst"])
        assert rel_err(f_col[0].cpu().numpy(), ref) < TOL
        ref_b = O.back_planesort(c["y"], c["Minv"], c["b"], c["src"], c["dst"], dims)
        assert rel_err(b_col[0].cpu().numpy(), ref_b) < TOL


def test_steep_case_mixes_both_walks():
    """The steep geometry really holds warps of both kinds: rows whose z
    slope exceeds 0.75 of the x-y slope (per-lane walk) and rows within it
    (column walk), in index space as the kernel decides."""
    c = _case("steep", seed=3)
    src, dst = c["src"].astype(np.float64), c["dst"].astype(np.float64)
    Mi = np.linalg.inv(c["M"].astype(np.float64))
    v = (dst - src) @ Mi.T
    ratio = np.abs(v[:, 2]) / np.maximum(np.abs(v[:, 0]), np.abs(v[:, 1]))
    hits = O.fwd_planesort(np.ones(tuple(c["n"]), np.float32), c["Minv"], c["b"], c["src"], c["dst"]) > 0
    assert (hits & (ratio > 0.75)).mean() > 0.05 and (hits & (ratio < 0.75)).mean() > 0.05
