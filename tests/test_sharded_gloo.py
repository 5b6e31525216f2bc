"""Ray-sharded projector logic across ranks on the CPU: world size 2 and 3
over gloo with a dense stand-in projector (the collectives, the partition,
uneven shards and the autograd path), and the partition itself.  The GPU
kernels under it are covered by the single-rank NCCL test in
test_gpu_sharded.py (this machine has no GPU and the GPU runs have one)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp
from torch import nn

from ct_laboratory_b200.sharded import RaySharded3DProjector, shard_bounds


def test_shard_bounds():
    assert shard_bounds(10, 3) == [(0, 4), (4, 8), (8, 10)]
    assert shard_bounds(12, 4, align=3) == [(0, 3), (3, 6), (6, 9), (9, 12)]
    assert shard_bounds(9, 2, align=3) == [(0, 6), (6, 9)]
    assert shard_bounds(3, 4) == [(0, 1), (1, 2), (2, 3), (3, 3)]
    with pytest.raises(ValueError):
        shard_bounds(10, 2, align=3)


class Rows(nn.Module):
    """Rows [lo, hi) of a dense operator on [n_x, n_y, n_z] volumes (batched)."""

    def __init__(self, A, lo, hi, shape):
        super().__init__()
        self.A, self.shape = A[lo:hi], shape
        self.n_x, self.n_y, self.n_z = shape

    def forward_project(self, v):
        flat = v.reshape(-1, self.A.shape[1])
        out = flat @ self.A.t()
        return out[0] if v.dim() == 3 else out

    def back_project(self, s):
        out = (s.reshape(-1, self.A.shape[0]) @ self.A).reshape(-1, *self.shape)
        return out[0] if s.dim() == 1 else out


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        shape, n_ray = (3, 4, 2), 11
        g = torch.Generator().manual_seed(0)
        A = torch.rand(n_ray, 24, generator=g, dtype=torch.float64)
        x = torch.rand(*shape, generator=g, dtype=torch.float64)
        y = torch.rand(n_ray, generator=g, dtype=torch.float64)
        p = RaySharded3DProjector(lambda lo, hi: Rows(A, lo, hi, shape), n_ray=n_ray)
        errs = []
        errs.append(float((p.forward_project(x) - A @ x.reshape(-1)).abs().max()))
        errs.append(float((p.back_project(y) - (y @ A).reshape(shape)).abs().max()))
        # a rank's own shard of the sinogram is accepted too
        errs.append(float((p.back_project(y[p.lo:p.hi]) - (y @ A).reshape(shape)).abs().max()))
        xb = torch.rand(2, *shape, generator=g, dtype=torch.float64)  # batched volumes
        errs.append(float((p.forward_project(xb) - xb.reshape(2, -1) @ A.t()).abs().max()))
        xr = x.clone().requires_grad_(True)
        w = torch.rand(n_ray, generator=g, dtype=torch.float64)
        (p(xr) * w).sum().backward()
        errs.append(float((xr.grad - (w @ A).reshape(shape)).abs().max()))
        local = RaySharded3DProjector(lambda lo, hi: Rows(A, lo, hi, shape), n_ray=n_ray, gather_sinogram=False)
        errs.append(float((local.forward_project(x) - (A @ x.reshape(-1))[local.lo:local.hi]).abs().max()))
        # equal shards (12 rays over 2 or 3 ranks): the gathered buffer is the sinogram itself
        A12 = torch.rand(12, 24, generator=g, dtype=torch.float64)
        p12 = RaySharded3DProjector(lambda lo, hi: Rows(A12, lo, hi, shape), n_ray=12)
        errs.append(float((p12.forward_project(x) - A12 @ x.reshape(-1)).abs().max()))
        errs.append(float((p12.forward_project(xb) - xb.reshape(2, -1) @ A12.t()).abs().max()))
        q.put((rank, max(errs)))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_projector_over_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(timeout=120)
    assert all(pr.exitcode == 0 for pr in procs), [pr.exitcode for pr in procs]
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert [r for r, _ in res] == list(range(world))
    assert max(e for _, e in res) < 1e-12
