"""Count the in-volume Siddon segments of a workload with the FP64 oracle
(test infrastructure; run once per workload, the result is frozen in
bench.py as the algorithmic-byte basis).

    python oracle/count_segments.py cone256|fan256|batch64

Counts, over all rays, the segments between consecutive plane parameters
whose midpoint voxel is inside the grid and whose length is > 0, under the
reference torch path's rules (ct_projector_3d_torch.py:219-271).
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from ct_laboratory_b200.workloads import WORKLOADS  # noqa: E402
from oracle import oracle as O  # noqa: E402


def count_batch(w):
    """Sum over the scans of a multi-scan workload (2-D)."""
    t0 = time.time()
    total = n_ray = 0
    for p in w.projectors("cpu"):
        Mi = np.linalg.inv(p.M.numpy().astype(np.float64))
        total += O.count_segments([p.n_row, p.n_col], Mi, p.b.numpy(), p.src.numpy(), p.dst.numpy(),
                                  dtype=np.float64)
        n_ray += p.src.shape[0]
    print(f"{w.name}: n_ray={n_ray} segments={total} mean={total / n_ray:.4f} "
          f"({time.time() - t0:.1f} s, {O.max_threads()} threads)")


def main():
    w = WORKLOADS[sys.argv[1] if len(sys.argv) > 1 else "cone256"]
    if hasattr(w, "projectors"):
        return count_batch(w)
    src, dst, M, b = w.geometry()
    src, dst = src.numpy(), dst.numpy()
    Mi = np.linalg.inv(M.numpy().astype(np.float64))
    t0 = time.time()
    total = 0
    chunk = 1 << 21
    for s in range(0, src.shape[0], chunk):
        total += O.count_segments(list(w.n), Mi, b.numpy(), src[s:s + chunk], dst[s:s + chunk], dtype=np.float64)
    print(f"{w.name}: n_ray={src.shape[0]} segments={total} mean={total / src.shape[0]:.4f} "
          f"({time.time() - t0:.1f} s, {O.max_threads()} threads)")


if __name__ == "__main__":
    main()
