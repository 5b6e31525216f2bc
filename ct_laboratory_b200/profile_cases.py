"""Small, fixed GPU cases for profiling the projector kernels with ncu.

    python -m ct_laboratory_b200.profile_cases static512-v24
    python -m ct_laboratory_b200.profile_cases batch64

Each case builds its inputs, then runs its kernels twice (a warm round and a
round to capture), and prints one line.  The inputs stay a few GB at most so
that a full ncu capture of a launch ends in a minute or two.

* ``static512-v24``: the static512 StaticCT ring (512^2 x 64 voxels over
  400 x 60 mm, 48 modules of 48 x 16 cells, 16 lit per source) cut to its
  first 24 of 240 views (294,912 rays).  Per round: the crossing-rule column
  walk in 16-lane groups (forward, adjoint), then the uint16-table forward
  and adjoint (the table built and compressed once, the float table freed).
* ``batch64``: the 64 uneven 2-D scans of the batched workload in one
  persistent launch per direction, forward with grid64 tiles of 256
  threads and adjoint with flat tiles of 128 threads (the autotuner's
  picks on a B200), image-sized scratch for the transposed 2-D adjoint.
"""
from __future__ import annotations

import sys

import torch


def static512_v24(device="cuda"):
    from . import _C
    from . import _native as N
    from .tomography import staticct_ray_tiling
    from .tomography._common import voxel_diag_len
    from .workloads import WORKLOADS
    w = WORKLOADS["static512"]
    dev = torch.device(device)
    p = w.projector(dev)
    nx, ny, nz = w.n
    per_view = w.modules_per_source * w.det_nx * w.det_ny
    n_keep = 24 * per_view
    src, dst = p.src[:n_keep].contiguous(), p.dst[:n_keep].contiguous()
    b, Mi = p.b, torch.inverse(p.M).contiguous()
    x = w.phantom(device=dev)
    y = torch.rand(n_keep, device=dev, generator=torch.Generator(device=dev).manual_seed(1))
    col16 = staticct_ray_tiling(n_keep // (w.det_nx * w.det_ny), w.det_nx, w.det_ny, voxel_rule=N.VOXEL_CROSSING)
    with torch.no_grad():
        tv = _C.compute_intersections_3d(nx, ny, nz, src, dst, Mi, b)
        u16, st, sc = _C.compress_tvals_3d_cuda(tv, src, dst, voxel_diag_len(p.M))
        del tv
        for _ in range(2):
            _C.forward_project_3d_on_the_fly_cuda(x, src, dst, Mi, b, tiling=col16)
            _C.back_project_3d_on_the_fly_cuda(y, src, dst, Mi, b, nx, ny, nz, tiling=col16)
            _C.forward_project_3d_compressed_cuda(x, u16, st, sc, src, dst, Mi, b)
            _C.back_project_3d_compressed_cuda(y, u16, st, sc, src, dst, Mi, b, nx, ny, nz)
    torch.cuda.synchronize(dev)
    return f"static512-v24: {n_keep} rays, uint16 table {u16.numel() * 2} bytes"


def batch64(device="cuda"):
    from .batched import ScanBatch
    from .workloads import WORKLOADS
    dev = torch.device(device)
    w = WORKLOADS["batch64"]
    batch = ScanBatch(w.projectors(dev), block_threads=128, kind="flat")
    batch.configure(block_threads=256, kind="grid64", direction="fwd", mode="persistent")
    batch.configure(block_threads=128, kind="flat", direction="adj", mode="persistent")
    g = torch.Generator(device=dev).manual_seed(2)
    for img, ph in zip(batch.images_in, w.phantoms(device=dev)):
        img.copy_(ph)
    for s in batch.sinos_in:
        s.copy_(torch.rand(s.shape, device=dev, generator=g))
    with torch.no_grad():
        for _ in range(2):
            batch.forward()
            batch.back()
    torch.cuda.synchronize(dev)
    return f"batch64: {len(batch.projectors)} scans, forward {batch.config}, adjoint {batch.config_adj}"


CASES = {"static512-v24": static512_v24, "batch64": batch64}


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 1 or argv[0] not in CASES:
        print(f"usage: python -m ct_laboratory_b200.profile_cases {{{','.join(CASES)}}}", file=sys.stderr)
        return 2
    if not torch.cuda.is_available():
        print("profile_cases: needs a CUDA device", file=sys.stderr)
        return 1
    print(CASES[argv[0]]())
    return 0


if __name__ == "__main__":
    sys.exit(main())
