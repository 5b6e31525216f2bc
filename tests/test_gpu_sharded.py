"""The ray-sharded projector on the GPU kernels: a single NCCL rank (this
run has one GPU) holding the whole cone-beam scan through the sharded path
(view-aligned slicing with the detector tiling, all-gather, all-reduce,
autograd) against the plain module.  Multi-rank logic: test_sharded_gloo.py."""
import os
import socket

import pytest
import torch
import torch.distributed as dist

from conftest import rel_err

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")


@pytest.fixture(scope="module")
def nccl_group():
    started = False
    if not dist.is_initialized():
        with socket.socket() as s:
            s.bind(("127.0.0.1", 0))
            port = s.getsockname()[1]
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        torch.cuda.set_device(0)
        dist.init_process_group("nccl", rank=0, world_size=1)
        started = True
    yield
    if started:
        dist.destroy_process_group()


def test_single_rank_sharded_cone_matches_module(nccl_group):
    from ct_laboratory_b200 import ConeBeam3DProjector
    from ct_laboratory_b200.sharded import RaySharded3DProjector, _slice_module
    p = ConeBeam3DProjector(24, 20, 16, n_view=9, det_nx=32, det_ny=24, sid=100.0, sdd=150.0, det_spacing=0.8,
                            voxel_size=0.5, voxel_rule=1, device=DEV)
    sp = RaySharded3DProjector(p)
    assert sp.bounds == [(0, p.src.shape[0])] and sp.local.ray_tiling.n_view == 9
    g = torch.Generator(device=DEV).manual_seed(0)
    x = torch.rand(24, 20, 16, generator=g, device=DEV)
    y = torch.rand(p.src.shape[0], generator=g, device=DEV)
    assert torch.equal(sp.forward_project(x), p.forward_project(x))
    assert rel_err(sp.back_project(y).cpu().numpy(), p.back_project(y).cpu().numpy()) < 1e-5
    xr = x.clone().requires_grad_(True)
    (sp(xr) * y).sum().backward()
    assert rel_err(xr.grad.cpu().numpy(), p.back_project(y).cpu().numpy()) < 1e-5
    # a view-aligned slice keeps the column-walk tiling and the same rays
    per_view = 32 * 24
    part = _slice_module(p, 3 * per_view, 7 * per_view)
    assert part.ray_tiling.n_view == 4
    assert torch.equal(part.forward_project(x), p.forward_project(x)[3 * per_view:7 * per_view])
