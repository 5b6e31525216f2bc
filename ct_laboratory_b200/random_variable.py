"""Random variables used by MAP reconstruction (likelihoods and priors).

Same classes, constructor arguments and semantics as the reference's
random_variable area (ct_laboratory/random_variable/{core,gaussian,poisson,
image_energies}.py): a likelihood is a ConditionalRandomVariable p(y | x)
evaluated at the measurements, a prior an unconditional RandomVariable p(x).
The forward operator enters as a closure (typically a projector's
``forward_project``), so autograd differentiates through the projector's
hand-written adjoint.

Reference files: core.py:131-196 (base classes), gaussian.py:6-80,
poisson.py:6-47 (Beer-Lambert photon counting, rate = I0 exp(-op(x))),
image_energies.py:12-29 (quadratic smoothness, non-periodic torch.diff).
"""
from __future__ import annotations

import torch
from torch import nn

__all__ = ["RandomVariable", "ConditionalRandomVariable", "DiagonalGaussianRandomVariable",
           "ConditionalGaussianRandomVariable", "LinearGaussianRandomVariable", "PoissonRandomVariable",
           "ConditionalPoissonRandomVariable", "BeerLambertPoissonRandomVariable",
           "QuadraticSmoothnessRandomVariable", "TotalVariationRandomVariable"]


class RandomVariable(nn.Module):
    """Unconditional random variable: log_prob / sample / score."""

    normalized = True

    def log_prob(self, x):  # pragma: no cover - abstract
        raise NotImplementedError

    def log_pdf(self, x):
        return self.log_prob(x)

    def sample(self, *args, **kwargs):  # pragma: no cover - abstract
        raise NotImplementedError(f"{type(self).__name__} does not implement sampling")

    def score(self, x):
        x = x.detach().requires_grad_(True)
        (grad,) = torch.autograd.grad(self.log_prob(x), x, create_graph=True)
        return grad

    def forward(self, x):
        return self.log_prob(x)


class ConditionalRandomVariable(nn.Module):
    """Family p(x | given); subclasses override evaluate() or log_prob()."""

    normalized = True

    def evaluate(self, given):  # pragma: no cover - abstract
        raise NotImplementedError

    def log_prob(self, x, given):
        return self.evaluate(given).log_prob(x)

    def log_pdf(self, x, given):
        return self.log_prob(x, given)

    def sample(self, given, *args, **kwargs):
        return self.evaluate(given).sample(*args, **kwargs)

    def score(self, x, given):
        x = x.detach().requires_grad_(True)
        (grad,) = torch.autograd.grad(self.log_prob(x, given), x, create_graph=True)
        return grad

    def forward(self, x, given):
        return self.log_prob(x, given)


class DiagonalGaussianRandomVariable(RandomVariable):
    """x ~ N(mu, diag(var))."""

    def __init__(self, mu, var=1.0):
        super().__init__()
        mu = torch.as_tensor(mu)
        var = torch.as_tensor(var, dtype=mu.dtype, device=mu.device)
        self.mu = mu
        self.var = torch.broadcast_to(var, mu.shape).contiguous()

    def _dist(self):
        return torch.distributions.Normal(self.mu, self.var.sqrt(), validate_args=False)

    def log_prob(self, x):
        return self._dist().log_prob(x).sum()

    def sample(self, sample_shape=torch.Size()):
        return self._dist().sample(sample_shape)

    def score(self, x):
        return (self.mu - x) / self.var


class ConditionalGaussianRandomVariable(ConditionalRandomVariable):
    """x | given ~ N(mean_fn(given), diag(var_fn(given)))."""

    def __init__(self, mean_fn, var_fn=1.0):
        super().__init__()
        self.mean_fn = mean_fn
        self.var_fn = var_fn if callable(var_fn) else (lambda given, v=var_fn: v)

    def evaluate(self, given):
        return DiagonalGaussianRandomVariable(self.mean_fn(given), self.var_fn(given))


class LinearGaussianRandomVariable(ConditionalGaussianRandomVariable):
    """y | x ~ N(op(x), diag(var)) for a linear operator closure."""

    def __init__(self, op, var=1.0):
        super().__init__(mean_fn=lambda x: op(x), var_fn=var)
        self.op = op


class PoissonRandomVariable(RandomVariable):
    """counts ~ Poisson(rate)."""

    def __init__(self, rate):
        super().__init__()
        self.register_buffer("rate", torch.as_tensor(rate))

    def _dist(self):
        return torch.distributions.Poisson(self.rate)

    def log_prob(self, x):
        return self._dist().log_prob(x).sum()

    def sample(self, sample_shape=torch.Size()):
        return self._dist().sample(sample_shape)


class ConditionalPoissonRandomVariable(ConditionalRandomVariable):
    """counts | x ~ Poisson(max(rate_fn(x), eps))."""

    def __init__(self, rate_fn, eps=1e-12):
        super().__init__()
        self.rate_fn = rate_fn
        self.eps = eps

    def evaluate(self, given):
        return PoissonRandomVariable(torch.clamp(self.rate_fn(given), min=self.eps))


class BeerLambertPoissonRandomVariable(ConditionalPoissonRandomVariable):
    """Photon-counting CT: counts | x ~ Poisson(I0 exp(-op(x)))."""

    def __init__(self, op, I0=1e6, eps=1e-12):
        super().__init__(rate_fn=lambda x: I0 * torch.exp(-op(x)), eps=eps)
        self.op = op
        self.I0 = float(I0)


def _neighbor_diffs(volume):
    for d in range(volume.dim()):
        yield torch.diff(volume, dim=d)


class QuadraticSmoothnessRandomVariable(RandomVariable):
    """log p(x) = -(w/2) ||grad x||^2 with non-periodic finite differences."""

    normalized = False

    def __init__(self, weight=1.0):
        super().__init__()
        self.weight = float(weight)

    def log_prob(self, x):
        energy = sum(d.pow(2).sum() for d in _neighbor_diffs(x))
        return -0.5 * self.weight * energy


class TotalVariationRandomVariable(RandomVariable):
    """log p(x) = -w TV(x), anisotropic."""

    normalized = False

    def __init__(self, weight=1.0):
        super().__init__()
        self.weight = float(weight)

    def log_prob(self, x):
        energy = sum(d.abs().sum() for d in _neighbor_diffs(x))
        return -self.weight * energy
