"""Preconditioners for the MAP estimator.

Contract of the reference's ct_laboratory/optimization/preconditioner.py:
a preconditioner is an ``nn.Module`` P applying a symmetric positive-definite
linear map (``forward``) and its inverse (``inverse``), and a class that
leaves either one unimplemented is refused with a TypeError as soon as it is
defined, not when it is first used.
"""
from __future__ import annotations

import torch
from torch import nn

__all__ = ["Preconditioner", "IdentityPreconditioner", "DiagonalPreconditioner"]

_DIRECTIONS = ("forward", "inverse")


class Preconditioner(nn.Module):
    """Base class: subclasses provide ``forward(x) = P x`` and
    ``inverse(x) = P^-1 x``."""

    def __init_subclass__(cls, **kwargs):
        super().__init_subclass__(**kwargs)
        # The class that supplies each direction is the first one along the
        # MRO defining it; reaching this base class means nobody did.
        for name in _DIRECTIONS:
            owner = next(c for c in cls.__mro__ if name in vars(c))
            if owner is Preconditioner or owner is nn.Module:
                raise TypeError(f"{cls.__name__} is not a complete preconditioner: it has no {name}() "
                                f"(a Preconditioner must define both {' and '.join(_DIRECTIONS)})")

    def forward(self, x):  # pragma: no cover - overridden by every concrete class
        raise NotImplementedError

    def inverse(self, x):  # pragma: no cover - overridden by every concrete class
        raise NotImplementedError

    def twice(self, x):
        """P(P(x)), the MAP estimator's step direction from a gradient; a
        subclass may give it in one pass."""
        return self(self(x))


class IdentityPreconditioner(Preconditioner):
    """P = I."""

    def forward(self, x):
        return x

    def inverse(self, x):
        return x


class DiagonalPreconditioner(Preconditioner):
    """P = diag(scale), scale > 0 elementwise (a tensor or a scalar)."""

    def __init__(self, scale):
        super().__init__()
        scale = torch.as_tensor(scale)
        if bool((scale <= 0).any()):
            raise ValueError("DiagonalPreconditioner needs a positive scale")
        self.register_buffer("scale", scale)

    def forward(self, x):
        return torch.mul(x, self.scale)

    def inverse(self, x):
        return torch.div(x, self.scale)
