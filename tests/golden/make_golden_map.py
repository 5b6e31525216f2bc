"""Golden MAP reconstructions from the reference's own estimator.

    python tests/golden/make_golden_map.py      # needs the reference checkout

Runs, on the CPU with the reference's torch projector, the reference's
MaximumAPosterioriEstimator with its BeerLambertPoissonRandomVariable
likelihood and QuadraticSmoothnessRandomVariable prior, preconditioned by its
SparseEigenDecomposition (subspace solver) -> SparseEigenImagePreconditioner,
on a small seeded cone-beam problem, and stores the measurements, the
eigen-basis and the reconstructions as tests/golden/map_cone.npz.
"""
from __future__ import annotations

import importlib
import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.reference_path import reference_root  # noqa: E402

REF = reference_root(required=True)

SHAPE = (16, 16, 8)
VOXEL = 0.8
GEOM = dict(n_view=24, det_nx=24, det_ny=12, sid=100.0, sdd=150.0, det_spacing=0.9)
I0 = 1e5
PRIOR_W = 1e-2
K = 8
N_ITERS = 50
LR_PRECOND = 2e-5
LR_PLAIN = 1e-8


def load_reference():
    pkg_dir = os.path.join(REF, "ct_laboratory")
    root = types.ModuleType("ct_laboratory")
    root.__path__ = [pkg_dir]
    sys.modules["ct_laboratory"] = root
    sys.modules["ct_laboratory._C"] = types.ModuleType("ct_laboratory._C")
    tomo = types.ModuleType("ct_laboratory.tomography")
    tomo.__path__ = [os.path.join(pkg_dir, "tomography")]
    sys.modules["ct_laboratory.tomography"] = tomo
    names = ["tomography.ct_projector_3d_module", "tomography.conebeam_projector_3d",
             "tomography.standard_image_transform", "random_variable", "optimization", "bayesian_estimation",
             "sparse_eigen_preconditioner"]
    return {n.split(".")[-1]: importlib.import_module("ct_laboratory." + n) for n in names}


def phantom(seed=3):
    g = torch.Generator().manual_seed(seed)
    axes = [torch.arange(n, dtype=torch.float32) / n - 0.5 for n in SHAPE]
    X, Y, Z = torch.meshgrid(*axes, indexing="ij")
    vol = torch.zeros(SHAPE)
    for _ in range(4):
        c = (torch.rand(3, generator=g) - 0.5) * 0.4
        a = torch.rand(3, generator=g) * 0.25 + 0.12
        inside = ((X - c[0]) / a[0]) ** 2 + ((Y - c[1]) / a[1]) ** 2 + ((Z - c[2]) / a[2]) ** 2 <= 1
        vol += 0.01 * torch.rand(1, generator=g) * inside.float()
    return (vol + 0.005).contiguous()


def main():
    torch.set_num_threads(1)
    m = load_reference()
    src, dst = m["conebeam_projector_3d"].build_conebeam_3d_geometry(**GEOM)
    M, b = m["standard_image_transform"].standard_image_transform_3d(*SHAPE, VOXEL, VOXEL, VOXEL)
    proj = m["ct_projector_3d_module"].CTProjector3DModule(*SHAPE, M, b, src, dst, backend="torch",
                                                           device=torch.device("cpu"),
                                                           precomputed_intersections=True, use_compression=False)
    x_true = phantom()
    with torch.no_grad():
        line = proj.forward_project(x_true)
    g = torch.Generator().manual_seed(5)
    y = torch.poisson(I0 * torch.exp(-line), generator=g)

    rv, opt, be, sep = m["random_variable"], m["optimization"], m["bayesian_estimation"], \
        m["sparse_eigen_preconditioner"]
    dec = sep.SparseEigenDecomposition(proj, k=K)
    dec.compute_weights(method="subspace", n_iters=30, seed=0, use_tqdm=False, compute_projection_basis=False)
    P = dec.to_image_preconditioner()

    def run(preconditioner, lr):
        lik = rv.BeerLambertPoissonRandomVariable(op=proj.forward_project, I0=I0)
        prior = rv.QuadraticSmoothnessRandomVariable(weight=PRIOR_W)
        est = be.MaximumAPosterioriEstimator(lik, prior, measurements=y, x_init=torch.zeros(SHAPE),
                                             preconditioner=preconditioner, lr=lr)
        losses = [est.step()[0] for _ in range(N_ITERS)]
        return est.x.numpy().copy(), np.array(losses)

    x_pre, loss_pre = run(P, LR_PRECOND)
    x_plain, loss_plain = run(None, LR_PLAIN)
    np.savez_compressed(os.path.join(HERE, "map_cone.npz"), shape=np.array(SHAPE), voxel=VOXEL, I0=I0,
                        prior_w=PRIOR_W, k=K, n_iters=N_ITERS, lr_pre=LR_PRECOND, lr_plain=LR_PLAIN,
                        x_true=x_true.numpy(), y=y.numpy(), s=dec.s.numpy(), v=dec.v.numpy(),
                        x_pre=x_pre, loss_pre=loss_pre, x_plain=x_plain, loss_plain=loss_plain,
                        **{f"geom_{k}": v for k, v in GEOM.items()})
    rel = lambda a: float(np.linalg.norm(a - x_true.numpy()) / np.linalg.norm(x_true.numpy()))  # noqa: E731
    print(f"eigenvalues {dec.s.numpy() ** 2}")
    print(f"preconditioned: loss {loss_pre[0]:.6e} -> {loss_pre[-1]:.6e}, rel err vs truth {rel(x_pre):.4f}")
    print(f"plain:          loss {loss_plain[0]:.6e} -> {loss_plain[-1]:.6e}, rel err vs truth {rel(x_plain):.4f}")


if __name__ == "__main__":
    main()
