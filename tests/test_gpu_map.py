"""MAP reconstruction and the sparse-eigen preconditioner against the
reference's own estimator (tests/golden/map_cone.npz, made by
tests/golden/make_golden_map.py with the reference's CPU projector).

Bar: reconstructions within 1e-4 relative RMSE of the reference's."""
import numpy as np
import pytest
import torch

from conftest import load_golden

pytestmark = pytest.mark.gpu
DEV = "cuda"


def setup():
    from ct_laboratory_b200 import ConeBeam3DProjector
    g = load_golden("map_cone")
    shape = tuple(int(v) for v in g["shape"])
    geom = {k[5:]: (float(g[k]) if "sid" in k or "sdd" in k or "spacing" in k else int(g[k]))
            for k in g if k.startswith("geom_")}
    p = ConeBeam3DProjector(*shape, **geom, voxel_size=float(g["voxel"]), device=torch.device(DEV))
    return g, shape, p


def rel_rmse(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def loss_atol(g):
    """Float32 evaluation noise of the summed Poisson loss.

    The loss sums one term per ray, rate - y log(rate) + lgamma(y + 1), each
    about lgamma(I0) (~1e6 at I0 = 1e5) and cancelling to a total that is
    orders of magnitude smaller; float32 rounds every term and the running sum
    to 2^-23 of that scale, and the reference evaluated it on the CPU with its
    own log / lgamma and summation order.  The bound is n_terms * scale * 2^-23
    (a few hundred here); the reconstructions themselves are held to 1e-4."""
    y = np.asarray(g["y"], np.float64)
    scale = float(np.max(np.abs(y * np.log(np.maximum(y, 1.0)) - y))) + float(g["I0"])
    return y.size * scale * 2.0 ** -23


def run_map(g, shape, p, preconditioner, lr):
    from ct_laboratory_b200.bayesian_estimation import MaximumAPosterioriEstimator
    from ct_laboratory_b200.random_variable import BeerLambertPoissonRandomVariable, QuadraticSmoothnessRandomVariable
    lik = BeerLambertPoissonRandomVariable(op=p.forward_project, I0=float(g["I0"]))
    prior = QuadraticSmoothnessRandomVariable(weight=float(g["prior_w"]))
    y = torch.as_tensor(g["y"]).to(DEV)
    est = MaximumAPosterioriEstimator(lik, prior, measurements=y, x_init=torch.zeros(shape, device=DEV),
                                      preconditioner=preconditioner, lr=lr)
    x = est.estimate(num_iters=int(g["n_iters"]))
    return x.cpu().numpy(), np.array([h[0] for h in est.history])


def test_map_preconditioned_matches_reference():
    from ct_laboratory_b200.sparse_eigen_preconditioner import SparseEigenImagePreconditioner
    g, shape, p = setup()
    P = SparseEigenImagePreconditioner(torch.as_tensor(g["s"]).to(DEV), torch.as_tensor(g["v"]).to(DEV))
    x, losses = run_map(g, shape, p, P, float(g["lr_pre"]))
    assert rel_rmse(x, g["x_pre"]) <= 1e-4
    assert np.allclose(losses, g["loss_pre"], rtol=1e-4, atol=loss_atol(g))


def test_map_plain_matches_reference():
    g, shape, p = setup()
    x, losses = run_map(g, shape, p, None, float(g["lr_plain"]))
    assert rel_rmse(x, g["x_plain"]) <= 1e-4
    assert np.allclose(losses, g["loss_plain"], rtol=1e-4, atol=loss_atol(g))


@pytest.mark.parametrize("method", ["subspace", "lanczos", "eigsh"])
def test_eigen_solvers_match_reference_spectrum(method):
    from ct_laboratory_b200.sparse_eigen_preconditioner import SparseEigenDecomposition
    g, shape, p = setup()
    k = int(g["k"])
    dec = SparseEigenDecomposition(p, k=k)
    kw = dict(n_iters=60, seed=0) if method == "subspace" else dict(tol=1e-6, seed=0)
    dec.compute_weights(method=method, **kw)
    ref = g["s"].astype(np.float64) ** 2
    got = dec.eigenvalues.cpu().numpy().astype(np.float64)
    assert np.allclose(got, ref, rtol=2e-3), (got, ref)
    # eigen-residuals ||G v - s^2 v|| small, and p = A v stored
    V = dec.v
    GV = dec._gram_matmul(V)
    res = (GV - V * dec.eigenvalues[None, :]).norm(dim=0) / dec.eigenvalues
    assert float(res.max()) < 5e-2
    assert dec.p.shape == (p.src.shape[0], k)


def test_projection_preconditioner_equals_image_preconditioner():
    from ct_laboratory_b200.sparse_eigen_preconditioner import SparseEigenDecomposition
    g, shape, p = setup()
    dec = SparseEigenDecomposition(p, k=8)
    dec.compute_weights(method="lanczos", tol=1e-7)
    Pi, Pp = dec.to_image_preconditioner(), dec.to_projection_preconditioner()
    x = torch.rand(int(np.prod(shape)), device=DEV)
    a, b = Pi(x), Pp(x)
    assert float((a - b).norm() / a.norm()) < 1e-3
    assert float((Pi.inverse(Pi(x)) - x).norm() / x.norm()) < 1e-4


def test_poisson_gradient_finite_differences():
    """Autograd gradient of -log p(y|x) - w log p(x) (through the projector's
    hand-written adjoint) against central differences, step 1e-3, 16 seeded
    voxels."""
    from ct_laboratory_b200.random_variable import BeerLambertPoissonRandomVariable, QuadraticSmoothnessRandomVariable
    g, shape, p = setup()
    lik = BeerLambertPoissonRandomVariable(op=p.forward_project, I0=float(g["I0"]))
    prior = QuadraticSmoothnessRandomVariable(weight=float(g["prior_w"]))
    y = torch.as_tensor(g["y"]).to(DEV)
    x0 = torch.as_tensor(g["x_true"]).to(DEV)

    def loss(x):
        return -(lik.log_prob(y, x) + prior.log_prob(x))

    xg = x0.clone().requires_grad_(True)
    loss(xg).backward()
    grad = xg.grad.double().flatten().cpu()
    I0 = float(g["I0"])
    w = float(g["prior_w"])
    yd = y.double()

    def loss64(x):
        # the same objective in float64 from the float32 projection (a
        # float32 sum of ~7k terms of size 1e5 would drown a 1e-3 step)
        rate = I0 * torch.exp(-p.forward_project(x).double())
        nll = (rate - yd * torch.log(rate) + torch.lgamma(yd + 1)).sum()
        xd = x.double()
        energy = sum((torch.diff(xd, dim=d) ** 2).sum() for d in range(3))
        return float(nll + 0.5 * w * energy)

    gen = torch.Generator().manual_seed(0)
    idx = torch.randperm(x0.numel(), generator=gen)[:16]
    h = 1e-3
    with torch.no_grad():
        for i in idx.tolist():
            e = torch.zeros(x0.numel(), device=DEV)
            e[i] = h
            e = e.view(shape)
            fd = (loss64(x0 + e) - loss64(x0 - e)) / (2 * h)
            assert abs(fd - float(grad[i])) <= 1e-3 * abs(float(grad[i])) + 1e-3 * float(grad.abs().max()), \
                (i, fd, float(grad[i]))
