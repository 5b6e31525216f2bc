"""Preconditioner contract (reference: ct_laboratory/optimization/preconditioner.py:20-66).

A preconditioner is a symmetric positive-definite linear map P with both
directions implemented; a subclass that fails to override ``forward`` or
``inverse`` is rejected when the class is defined.
"""
from __future__ import annotations

import torch
from torch import nn

__all__ = ["Preconditioner", "IdentityPreconditioner", "DiagonalPreconditioner"]


class Preconditioner(nn.Module):
    def __init_subclass__(cls, **kwargs):
        super().__init_subclass__(**kwargs)
        for required in ("forward", "inverse"):
            impl = cls.__dict__.get(required)
            inherited = getattr(cls, required, None)
            if impl is None and (inherited is None or inherited in (Preconditioner.forward, Preconditioner.inverse)):
                raise TypeError(f"Preconditioner subclass {cls.__name__!r} must implement {required!r} "
                                "(both forward and inverse are required)")

    def forward(self, x):  # pragma: no cover - abstract
        raise NotImplementedError

    def inverse(self, x):  # pragma: no cover - abstract
        raise NotImplementedError


class IdentityPreconditioner(Preconditioner):
    def forward(self, x):
        return x

    def inverse(self, x):
        return x


class DiagonalPreconditioner(Preconditioner):
    def __init__(self, scale):
        super().__init__()
        scale = torch.as_tensor(scale)
        if torch.any(scale <= 0):
            raise ValueError("DiagonalPreconditioner scale must be positive")
        self.register_buffer("scale", scale)

    def forward(self, x):
        return x * self.scale

    def inverse(self, x):
        return x / self.scale
