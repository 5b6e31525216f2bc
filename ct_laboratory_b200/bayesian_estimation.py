"""MAP estimation: x* = argmin_x -log p(y | x) - w log p(x).

Contract of the reference's MaximumAPosterioriEstimator
(ct_laboratory/bayesian_estimation/map_estimator.py:28-135): the likelihood
is a ConditionalRandomVariable, the prior a RandomVariable, the
preconditioner a Preconditioner (identity by default); each step moves x
against the preconditioned gradient direction F g = P(P(g)), applied outside
autograd, with step size lr (ramped linearly over the first `warmup_iters`
steps when given, starting from 0 on the first step); ``step()`` returns
(loss, log_lik, log_prior) as floats and ``estimate()`` returns x.

Here the update is written out instead of going through torch.optim:
x <- x - lr_k * P(P(grad)), lr_k = lr * min(1, k / warmup_iters) on step k
(counting from 0), the same update and schedule as SGD under LambdaLR.
``estimate()`` keeps each step's losses on the device and reads them back
once at the end instead of synchronising three times per step.
"""
from __future__ import annotations

import time

import torch

from .optimization import IdentityPreconditioner, Preconditioner
from .random_variable import ConditionalRandomVariable, RandomVariable

__all__ = ["MaximumAPosterioriEstimator"]


def _expect(value, kind, what):
    if not isinstance(value, kind):
        raise TypeError(f"{what} must be a {kind.__name__}, not {type(value).__name__}")


class MaximumAPosterioriEstimator:
    def __init__(self, likelihood, prior, measurements, x_init, preconditioner=None, lr=1.0, warmup_iters=None,
                 prior_weight=1.0):
        _expect(likelihood, ConditionalRandomVariable, "likelihood")
        _expect(prior, RandomVariable, "prior")
        preconditioner = IdentityPreconditioner() if preconditioner is None else preconditioner
        _expect(preconditioner, Preconditioner, "preconditioner")
        self.likelihood = likelihood
        self.prior = prior
        self.measurements = measurements
        self.preconditioner = preconditioner
        self.prior_weight = float(prior_weight)
        self.lr = float(lr)
        self.warmup_iters = warmup_iters
        self.steps_taken = 0
        self._x = x_init.detach().clone()
        self.history = []

    @property
    def x(self):
        """The current estimate (shape of x_init)."""
        return self._x

    def learning_rate(self, k=None):
        """Step size of step k (default: the next step)."""
        k = self.steps_taken if k is None else k
        if self.warmup_iters is None:
            return self.lr
        return self.lr * min(1.0, float(k) / self.warmup_iters)

    def negative_log_posterior(self, x):
        """(-log p(y|x) - w log p(x), log p(y|x), log p(x))."""
        log_likelihood = self.likelihood.log_prob(self.measurements, x)
        log_prior = self.prior.log_prob(x)
        return -(log_likelihood + self.prior_weight * log_prior), log_likelihood, log_prior

    def _advance(self):
        """One step; returns the step's (loss, log_lik, log_prior) as one
        device tensor."""
        x = self._x.detach().requires_grad_(True)
        terms = self.negative_log_posterior(x)
        (grad,) = torch.autograd.grad(terms[0], x)
        with torch.no_grad():
            P = self.preconditioner
            twice = getattr(P, "twice", None)
            g = grad.reshape(-1)
            direction = (twice(g) if twice is not None else P(P(g))).reshape(grad.shape)
            self._x = x.detach().add_(direction, alpha=-self.learning_rate())
        self.steps_taken += 1
        return torch.stack([t.detach() for t in terms])

    def step(self):
        """One preconditioned gradient step; returns (loss, log_lik, log_prior)."""
        loss, log_lik, log_prior = self._advance().tolist()
        self.history.append([loss, log_lik, log_prior])
        return loss, log_lik, log_prior

    def estimate(self, num_iters=100, verbose=False, use_tqdm=False, print_every=1):
        """Run `num_iters` steps and return the estimate; every step's losses
        are appended to ``history``."""
        t0 = time.time()
        record = []
        for it in range(1, num_iters + 1):
            record.append(self._advance())
            if verbose and (it == 1 or it % print_every == 0):
                loss, log_lik, log_prior = record[-1].tolist()
                print(f"step {it:4d}: loss {loss:.4e}  -log p(y|x) {-log_lik:.4e}  -log p(x) {-log_prior:.4e}  "
                      f"({time.time() - t0:.2f} s)")
                t0 = time.time()
        if record:
            self.history.extend(torch.stack(record).cpu().tolist())
        return self.x
