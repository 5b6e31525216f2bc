"""The CPU oracle against the reference's own outputs (tests/golden, made by
tests/golden/make_golden.py from the reference's torch path) and its two
known answers.  CPU only."""
import numpy as np
import pytest

from conftest import load_golden, rel_err
from oracle import oracle as O

CASES_2D = ["kat2d", "fan2d", "static2d"]
CASES_3D = ["kat3d", "cone3d", "affine3d", "edge3d", "static3d"]
DIAGONAL = ["kat2d", "fan2d", "static2d", "kat3d", "cone3d", "edge3d", "static3d"]


@pytest.mark.parametrize("name", CASES_2D + CASES_3D)
def test_intersections(name):
    g = load_golden(name)
    tv = O.isect_torch(g["dims"], g["Minv"], g["b"], g["src"], g["dst"])
    if name in DIAGONAL:
        # diagonal affine: the index-space mapping is exact, so every value is
        assert np.array_equal(tv, g["tvals"])
    else:
        # non-diagonal: torch's matmul may fuse differently (1 ulp)
        fin = np.isfinite(g["tvals"])
        assert np.array_equal(fin, np.isfinite(tv))
        assert np.abs(tv[fin] - g["tvals"][fin]).max() < 1e-5


@pytest.mark.parametrize("name", CASES_2D + CASES_3D)
def test_forward_and_adjoint(name):
    g = load_golden(name)
    img = g["img"] if "img" in g else g["vol"]
    fwd = O.fwd_tvals_torch(img, g["tvals"], g["Minv"], g["b"], g["src"], g["dst"])
    back = O.back_tvals_torch(g["y"], g["tvals"], g["Minv"], g["b"], g["src"], g["dst"], g["dims"])
    otf = O.fwd_otf_torch(img, g["Minv"], g["b"], g["src"], g["dst"])
    assert rel_err(fwd, g["fwd"]) < 1e-6
    assert rel_err(back, g["back"]) < 1e-6
    tol = 2e-6 if name in DIAGONAL else 1e-5  # non-diagonal: matmul order differs by an ulp
    assert rel_err(otf, g["fwd"]) < tol
    otb = O.back_otf_torch(g["y"], g["Minv"], g["b"], g["src"], g["dst"], g["dims"])
    assert rel_err(otb, g["back"]) < tol


def test_known_answers():
    # python_examples/test_ct_projector_{2d,3d}_line_integral.py: "should equal 32.0"
    g2 = load_golden("kat2d")
    assert g2["fwd"][0] == np.float32(32.0)
    assert O.fwd_otf_torch(g2["img"], g2["Minv"], g2["b"], g2["src"], g2["dst"])[0] == np.float32(32.0)
    g3 = load_golden("kat3d")
    assert abs(float(g3["fwd"][0]) - 32.0) < 2e-5
    assert O.fwd_otf_torch(g3["vol"], g3["Minv"], g3["b"], g3["src"], g3["dst"])[0] == g3["fwd"][0]
    assert abs(float(O.fwd_planesort(g3["vol"], g3["Minv"], g3["b"], g3["src"], g3["dst"])[0]) - 32.0) < 2e-5


@pytest.mark.parametrize("name", ["cone3d", "affine3d"])
def test_uint16_codec_bit_exact(name):
    g = load_golden(name)
    vd = O.voxel_diag_len(g["M"])
    assert np.float32(vd) == g["voxel_diag"]
    u16, starts, scales = O.compress_torch(g["tvals"], g["src"], g["dst"], vd)
    assert np.array_equal(scales, g["scales"])
    assert np.array_equal(starts, g["starts"])
    assert np.array_equal(u16, g["u16"])
    dec = O.decompress_torch(g["u16"], g["starts"], g["scales"])
    assert np.array_equal(dec, g["decomp"])
    fc = O.fwd_tvals_torch(g["vol"], dec, g["Minv"], g["b"], g["src"], g["dst"])
    assert rel_err(fc, g["fwd_comp"]) < 1e-6


@pytest.mark.parametrize("name", CASES_3D)
def test_fp64_adjoint_identity(name):
    """<A x, y> = <x, A^T y> for the FP64 oracle (same tvals, same segments)."""
    g = load_golden(name)
    dims = g["dims"]
    tv = O.isect_torch(dims, np.linalg.inv(g["M"].astype(np.float64)), g["b"], g["src"], g["dst"],
                       dtype=np.float64)
    Mi = np.linalg.inv(g["M"].astype(np.float64))
    rng = np.random.default_rng(0)
    x = rng.random(tuple(dims))
    y = rng.random(g["src"].shape[0])
    ax = O.fwd_tvals_torch(x, tv, Mi, g["b"], g["src"], g["dst"], dtype=np.float64)
    aty = O.back_tvals_torch(y, tv, Mi, g["b"], g["src"], g["dst"], dims, dtype=np.float64)
    lhs, rhs = float(ax @ y), float((x * aty).sum())
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0)


def test_cuda_path_emulations_agree_with_torch_path():
    """The plane-sort and compressed-decode restatements stay within float
    rounding of the torch path on the golden geometries."""
    for name in ["cone3d", "static3d", "edge3d"]:
        g = load_golden(name)
        ps = O.fwd_planesort(g["vol"], g["Minv"], g["b"], g["src"], g["dst"])
        assert rel_err(ps, g["fwd"]) < 1e-5


@pytest.mark.parametrize("name", ["cone3d", "affine3d"])
def test_cuda_encoder_round_trip_on_unclamped_rows(name):
    """The reference CUDA encoder's stream decodes (start + k*scale, fused)
    to within half a step of every finite t on rows where no delta reached
    the 32000 clamp.  Rows that hit the clamp (plane hits far outside the
    volume, e.g. a source lying on a plane) carry a deficit: that is the
    reference's behaviour and is not corrected."""
    g = load_golden(name)
    u16, st, sc = O.compress_cuda(g["tvals"], g["src"], g["dst"], float(g["voxel_diag"]))
    k = np.cumsum(u16.astype(np.int64), axis=1).astype(np.float32)
    dec = (k.astype(np.float64) * sc[:, None].astype(np.float64) + st[:, None]).astype(np.float32)
    ok_rows = (u16.max(axis=1) < 32000) & np.isfinite(st)
    assert ok_rows.sum() > 0
    t = g["tvals"][ok_rows]
    fin = np.isfinite(t)
    err = np.abs(dec[ok_rows][fin] - t[fin]) / np.repeat(sc[ok_rows], fin.sum(axis=1))
    assert err.max() <= 0.6  # half a step plus float32 rounding of 1/scale and of t


def test_reference_adjoint_bug_is_visible_in_emulation():
    """The reference's on-the-fly 3-D adjoint receives M instead of M^-1
    (ct_projector_3d_cuda.py:209-210 then :319).  Emulating that with the
    plane-sort restatement breaks the adjoint identity at 0.5 mm voxels,
    while the correct M^-1 keeps it."""
    g = load_golden("cone3d")
    dims = (14, 12, 10)
    M = np.diag([0.5, 0.5, 0.5]).astype(np.float32)
    b = (-(np.array(dims) - 1) / 2.0 * 0.5).astype(np.float32)
    rng = np.random.default_rng(1)
    x = rng.random(dims).astype(np.float32)
    y = rng.random(g["src"].shape[0]).astype(np.float32)
    Mi = np.linalg.inv(M).astype(np.float32)
    ax = O.fwd_planesort(x, Mi, b, g["src"], g["dst"])
    good = O.back_planesort(y, Mi, b, g["src"], g["dst"], dims)
    bad = O.back_planesort(y, M, b, g["src"], g["dst"], dims)
    lhs = float(ax.astype(np.float64) @ y)
    assert abs(lhs - float((x * good).sum(dtype=np.float64))) < 1e-4 * lhs
    assert abs(lhs - float((x * bad).sum(dtype=np.float64))) > 0.1 * lhs
