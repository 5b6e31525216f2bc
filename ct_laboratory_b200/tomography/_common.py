"""Helpers shared by the function-level API and the modules."""
from __future__ import annotations

import torch

from .. import _native as N


def require_cuda(*tensors, what="inputs"):
    """The projector runs on CUDA devices only; there is no CPU path."""
    for t in tensors:
        if t is not None and isinstance(t, torch.Tensor) and not t.is_cuda:
            raise RuntimeError(f"ct_laboratory_b200: {what} must be CUDA tensors (got a {t.device} tensor); "
                               "this package has no CPU implementation")


def as_f32(t):
    return t if t.dtype == torch.float32 and t.is_contiguous() else t.to(torch.float32).contiguous()


def single_affine(M, b, n_ray=None):
    """The reference accepts per-ray stacks of M/b and uses the first one
    (ct_projector_3d_cuda.py:130-132, :263-265)."""
    if M.dim() > 2:
        M = M[0]
        b = b[0] if b.dim() > 1 else b
    return M, b


def inverse(M: torch.Tensor) -> torch.Tensor:
    """M^-1 (float32, contiguous) computed on M's device by the C ABI, with no
    host synchronisation.  Plays the part of the reference's
    _prepare_M_inv / _M_inv (ct_projector_3d_cuda.py:42-48,
    ct_projector_2d_cuda.py:6-8), including its TypeError for CPU input."""
    if not M.is_cuda:
        raise TypeError("M must be a CUDA tensor (got CPU)")
    Mc = as_f32(M)
    n = Mc.shape[-1]
    if Mc.shape != (n, n) or n not in (2, 3):
        raise RuntimeError(f"M must be 2x2 or 3x3 (got {tuple(M.shape)})")
    out = torch.empty_like(Mc)
    with torch.cuda.device(Mc.device):
        N.call("ctlab_invert_matrix", N.ptr(Mc), n, N.ptr(out), None, N.stream_of(Mc))
    return out


class InverseCache:
    """M^-1 of a module's M buffer, recomputed only when the buffer object,
    its device or its in-place version changes."""

    def __init__(self):
        self._key = None
        self._val = None

    def get(self, M: torch.Tensor) -> torch.Tensor:
        key = (id(M), M.device, M._version, tuple(M.shape))
        if self._key != key or self._val is None:
            self._val = inverse(M)
            self._key = key
            self._ref = M  # keep the keyed object alive so its id stays unique
        return self._val


def voxel_diag_len(M: torch.Tensor) -> float:
    """Longest body diagonal of a voxel, |M d| over the four diagonals, in the
    torch ops the reference uses (ct_projector_3d_cuda.py:97-104)."""
    if M.dim() > 2:
        M = M[0]
    diags = torch.tensor([[1, 1, 1], [1, 1, -1], [1, -1, 1], [-1, 1, 1]], device=M.device, dtype=M.dtype).t()
    return torch.norm(M @ diags, dim=0).max().item()
