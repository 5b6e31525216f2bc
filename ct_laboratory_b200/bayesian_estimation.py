"""MAP estimation: x* = argmax_x log p(y | x) + w log p(x).

Same contract as the reference's MaximumAPosterioriEstimator
(ct_laboratory/bayesian_estimation/map_estimator.py:28-135): SGD on x with
learning rate ``lr`` (optional linear warm-up), the raw gradient g replaced
by the preconditioned direction F g = P(P(g)) outside autograd, prior weight
``prior_weight``.  ``step()`` returns (loss, log_lik, log_prior) as floats
like the reference; ``estimate()`` runs the same steps without the three
host synchronisations per iteration that the reference's ``.item()`` calls
make, reading the losses back once at the end.
"""
from __future__ import annotations

import time

import torch

from .optimization import IdentityPreconditioner, Preconditioner
from .random_variable import ConditionalRandomVariable, RandomVariable

__all__ = ["MaximumAPosterioriEstimator"]


class MaximumAPosterioriEstimator:
    def __init__(self, likelihood, prior, measurements, x_init, preconditioner=None, lr=1.0, warmup_iters=None,
                 prior_weight=1.0):
        if not isinstance(likelihood, ConditionalRandomVariable):
            raise TypeError(f"likelihood must be a ConditionalRandomVariable (got {type(likelihood).__name__})")
        if not isinstance(prior, RandomVariable):
            raise TypeError(f"prior must be a RandomVariable (got {type(prior).__name__})")
        if preconditioner is None:
            preconditioner = IdentityPreconditioner()
        if not isinstance(preconditioner, Preconditioner):
            raise TypeError("preconditioner must be a ct_laboratory_b200.optimization.Preconditioner "
                            f"(got {type(preconditioner).__name__})")
        self.likelihood = likelihood
        self.prior = prior
        self.measurements = measurements
        self.preconditioner = preconditioner
        self.prior_weight = float(prior_weight)
        self._shape = x_init.shape
        self.x_var = x_init.detach().clone().requires_grad_(True)
        self.optimizer = torch.optim.SGD([self.x_var], lr=lr)
        self.scheduler = None
        if warmup_iters is not None:
            self.scheduler = torch.optim.lr_scheduler.LambdaLR(
                self.optimizer, lr_lambda=lambda it: min(1.0, float(it) / warmup_iters))
        self.history = []

    @property
    def x(self):
        return self.x_var.detach().reshape(self._shape)

    def negative_log_posterior(self, x):
        log_likelihood = self.likelihood.log_prob(self.measurements, x)
        log_prior = self.prior.log_prob(x)
        return -(log_likelihood + self.prior_weight * log_prior), log_likelihood, log_prior

    def _step(self):
        self.optimizer.zero_grad()
        loss, log_likelihood, log_prior = self.negative_log_posterior(self.x_var.reshape(self._shape))
        loss.backward()
        with torch.no_grad():
            g = self.x_var.grad.reshape(-1)
            direction = self.preconditioner(self.preconditioner(g))
            self.x_var.grad = direction.reshape(self.x_var.shape)
        self.optimizer.step()
        if self.scheduler is not None:
            self.scheduler.step()
        return loss.detach(), log_likelihood.detach(), log_prior.detach()

    def step(self):
        """One preconditioned gradient step; returns (loss, log_lik, log_prior)."""
        loss, ll, lp = self._step()
        return loss.item(), ll.item(), lp.item()

    def estimate(self, num_iters=100, verbose=False, use_tqdm=False, print_every=1):
        """Run ``num_iters`` steps and return the MAP estimate x*.  Losses of
        every step are kept in ``self.history`` (read back once at the end)."""
        t0 = time.time()
        losses = []
        for it in range(1, num_iters + 1):
            losses.append(torch.stack(self._step()))
            if verbose and (it % print_every == 0 or it == 1):
                loss, ll, lp = losses[-1].tolist()
                print(f"iter {it:04d}  -log_lik={-ll:.4e}  -log_prior={-lp:.4e}  loss={loss:.4e}  "
                      f"({time.time() - t0:.2f}s)")
                t0 = time.time()
        if losses:
            self.history.extend(torch.stack(losses).cpu().tolist())
        return self.x
