"""MultiRotationProjector window logic on the CPU (no projector kernel):
z-window bounds and padding against a restatement of the reference's rules
(tomography/ct_projector_3d_multirot.py:51-152, 258-310), and the adjoint
identity <F x, y> = <x, B y> with a dense stand-in projector."""
import numpy as np
import pytest
import torch
from torch import nn

from ct_laboratory_b200.tomography.ct_projector_3d_multirot import MultiRotationProjector


class DenseProjector(nn.Module):
    """A dense linear operator on [n_x, n_y, n_z] volumes (batched), with its transpose."""

    def __init__(self, shape, n_ray, seed=0):
        super().__init__()
        g = torch.Generator().manual_seed(seed)
        self.shape = shape
        self.n_x, self.n_y, self.n_z = shape
        self.A = torch.rand(n_ray, int(np.prod(shape)), generator=g, dtype=torch.float64)

    def forward(self, v):
        flat = v.reshape(-1, self.A.shape[1]).double()
        out = flat @ self.A.t()
        return out[0] if v.dim() == 3 else out

    def back_project(self, s):
        out = s.reshape(-1, self.A.shape[0]).double() @ self.A
        out = out.reshape(-1, *self.shape)
        return out[0] if s.dim() == 1 else out


def ref_bounds(z, n_rot, shift, n_win, center=None):
    c = (float(center) - 0.5) if center is not None else (z - 1) / 2.0
    out = []
    for i in range(n_rot):
        rc = c - (n_rot - 1) / 2.0 * shift + i * shift
        s = int(round(rc - (n_win - 1) / 2.0))
        out.append((s, s + n_win))
    return out


def ref_source(idx, z, mode, limit):
    """Source slice of window slice idx (None = zero) under the reference's rules."""
    if 0 <= idx < z:
        return idx
    if mode == "repeat":
        return min(max(idx, 0), z - 1)
    if mode == "reflect":
        if limit is not None and (idx < -limit or idx >= z + limit):
            return None
        k = idx
        while k < 0 or k >= z:
            k = -k if k < 0 else 2 * z - 2 - k
        return k
    return None


@pytest.mark.parametrize("center", [None, 3])
def test_window_bounds(center):
    m = MultiRotationProjector(None, n_rotations=5, shift_offset=2.5, n_z_window=6, scan_center_slice=center)
    assert [m._get_rotation_z_bounds(12, i) for i in range(5)] == ref_bounds(12, 5, 2.5, 6, center)


@pytest.mark.parametrize("mode,limit", [("repeat", None), ("reflect", None), ("reflect", 2), ("zeros", None)])
def test_window_padding(mode, limit):
    z = 7
    vol = torch.rand(3, 4, z, dtype=torch.float64)
    m = MultiRotationProjector(None, n_rotations=4, shift_offset=4.0, n_z_window=8, padding_mode=mode,
                               reflection_padding_slices=limit)
    for i in range(4):
        s, e = m._get_rotation_z_bounds(z, i)
        got = m._extract_volume_slice(vol, s, e)
        for k, idx in enumerate(range(s, e)):
            src = ref_source(idx, z, mode, limit)
            want = torch.zeros(3, 4, dtype=vol.dtype) if src is None else vol[..., src]
            assert torch.equal(got[..., k], want), (mode, i, idx)


@pytest.mark.parametrize("mode,limit", [("repeat", None), ("reflect", None), ("reflect", 1), ("zeros", None)])
def test_back_project_is_the_transpose(mode, limit):
    z = 9
    base = DenseProjector((3, 2, 5), n_ray=6, seed=1)
    m = MultiRotationProjector(base, n_rotations=4, shift_offset=3.0, n_z_window=5, padding_mode=mode,
                               reflection_padding_slices=limit)
    x = torch.rand(3, 2, z, dtype=torch.float64)
    y = torch.rand(6, 4, dtype=torch.float64)
    fx = m(x)
    assert fx.shape == (6, 4)
    bty = m.back_project(y, z)
    assert bty.shape == (3, 2, z)
    assert abs(float((fx * y).sum()) - float((x * bty).sum())) < 1e-9 * float((fx * y).sum())


def test_repeat_padding_gives_no_gradient_through_copies():
    z = 5
    base = DenseProjector((2, 2, 4), n_ray=3, seed=2)
    m = MultiRotationProjector(base, n_rotations=2, shift_offset=4.0, n_z_window=4, padding_mode="repeat")
    x = torch.rand(2, 2, z, dtype=torch.float64, requires_grad=True)
    m(x).sum().backward()
    # gradient equals the adjoint restricted to in-volume window slices
    y = torch.ones(3, 2, dtype=torch.float64)
    full = torch.zeros(2, 2, z, dtype=torch.float64)
    wins = base.back_project(y.t().contiguous())
    for i in range(2):
        s, e = m._get_rotation_z_bounds(z, i)
        for k, idx in enumerate(range(s, e)):
            if 0 <= idx < z:
                full[..., idx] += wins[i][..., k]
    assert torch.allclose(x.grad, full)
