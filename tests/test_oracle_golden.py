"""The oracle's restatements pinned to the reference: to its own generated
C++ (Harris, unsharp, local Laplacian; fixtures made by
tests/golden/make_golden.py) and, for the pipelines it ships no generated
code for (camera pipe, bilateral grid, pyramid blending), to its own DSL
specs evaluated point by point (fixtures made by
tests/golden/make_spec_golden.py)."""

import os

import numpy as np

import oracle.harris as OH
import oracle.unsharp as OU

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_harris_matches_reference_cpp():
    g = np.load(os.path.join(GOLD, "harris.npz"))
    ours = OH.harris(g["img"])
    ref = g["out"].astype(np.float64)
    # refHarris computes in float32: compare relative to the output scale
    assert np.abs(ours - ref).max() / np.abs(ref).max() < 1e-6
    # refHarris zero-fills; both leave the 2-pixel border at 0
    H, W = ref.shape
    mask = np.ones_like(ref, dtype=bool)
    mask[2:H - 1, 2:W - 1] = False
    assert np.all(ref[mask] == 0) and np.all(ours[mask] == 0)


def test_unsharp_matches_reference_cpp_on_defined_region():
    g = np.load(os.path.join(GOLD, "unsharp.npz"))
    u8 = g["img"]
    thr, w = float(g["threshold"]), float(g["weight"])
    planar = np.moveaxis(u8.astype(np.float32) / np.float32(255.0), 2, 0)
    ours = OU.unsharp(planar, thr, w)
    ref = np.moveaxis(g["out"], 2, 0).astype(np.float64)
    R, C = ref.shape[1:]
    xs, ys = OU.defined_region(R, C)
    m = OU.margin(planar, thr)[:, xs, ys] > 1e-6
    d = np.abs(ours[:, xs, ys] - ref[:, xs, ys])
    assert d[m].max() < 1e-5


def test_unsharp_convention_outside_defined_region():
    """Columns whose blur reaches uncomputed blurx points use 0 there."""
    img = OU.make_input(10, 12, seed=4)
    out = OU.unsharp(img, 0.001, 3.0)
    assert out.shape == (3, 10, 12)
    assert np.all(out[:, 9, :] == 0) and np.all(out[:, :, 11] == 0)


def test_clamped_pyramid_oracle_matches_reference_spec_inside():
    """The generalized (clamped) pyramid spec at L = 4 equals the
    reference's 4-level spec on the reference's output box, where no
    clamp is reached."""
    import oracle.pyramid as OP
    R, C = 157, 211
    img1, img2, mask = OP.make_inputs(R, C, seed=2)
    ref = OP.pyramid_blend(img1, img2, mask, L=4)
    gen = OP.pyramid_blend_clamped(img1, img2, mask, L=4)
    (x0, x1), (y0, y1) = OP.output_box(R, C)
    assert ref.shape == (3, x1 - x0 + 1, y1 - y0 + 1)
    assert np.abs(gen[:, x0:x1 + 1, y0:y1 + 1] - ref).max() < 1e-12


def test_laplacian_restatement_matches_reference_fixtures():
    """The float32 NumPy restatement of the local Laplacian reproduces the
    reference's compiled pipeline_laplacian exactly on the fixtures."""
    import oracle.laplacian as OL
    z = np.load(os.path.join(GOLD, "laplacian.npz"))
    for n in range(2):
        got = OL.local_laplacian(z['frame%d' % n], float(z['alpha']),
                                 float(z['beta']))
        assert np.array_equal(got, z['out%d' % n])


# ---------------------------------------------------------------------------
# Restatements of the pipelines the reference ships no generated code for,
# pinned to the reference's own DSL specs evaluated point by point
# (fixtures written by tests/golden/make_spec_golden.py).

def test_campipe_restatement_matches_reference_spec():
    """oracle/campipe.c equals the reference's camera_pipe spec evaluated
    with C semantics, byte for byte, at two parameter sets; its const
    tables equal the spec's matrix and all 65536 curve entries."""
    import oracle.campipe as OC
    z = np.load(os.path.join(GOLD, "campipe_spec.npz"))
    for n in range(2):
        kelvin, contrast, gamma = (float(v) for v in z['params%d' % n])
        got = OC.campipe(z['img%d' % n], kelvin, contrast, gamma)
        assert np.array_equal(got, z['out%d' % n])
    mat, lut = OC.tables(*(float(v) for v in z['params0']))
    assert np.array_equal(mat, z['matrix'])
    assert np.array_equal(lut, z['lut'])


def test_bilateral_restatement_matches_reference_spec():
    """oracle/bilateral.py equals the reference's bilateral_grid spec in
    FP64 (bins as compiled) to FP64 round-off; the reference's own float
    arithmetic stays within 1e-5 of it."""
    import oracle.bilateral as OB
    z = np.load(os.path.join(GOLD, "bilateral_spec.npz"))
    for n in range(2):
        got = OB.bilateral(z['img%d' % n])
        assert np.abs(got - z['fp64%d' % n]).max() <= 1e-12
        assert np.abs(got - z['f32%d' % n]).max() <= 1e-5


def test_pyramid_restatement_matches_reference_spec():
    """oracle/pyramid.py (L = 4) equals the reference's pyramid_blending
    spec in FP64 over the spec's output box; the reference's own float
    arithmetic stays within 1e-6 of it."""
    import oracle.pyramid as OP
    z = np.load(os.path.join(GOLD, "pyramid_spec.npz"))
    for n in range(2):
        R, C = (int(v) for v in z['shape%d' % n])
        i1, i2, m = OP.make_inputs(R, C, seed=R)
        got = OP.pyramid_blend(i1, i2, m)
        (x0, x1), (y0, y1) = OP.output_box(R, C)
        assert tuple(z['lo%d' % n]) == (0, x0, y0)
        assert got.shape == z['fp64%d' % n].shape
        assert np.abs(got - z['fp64%d' % n]).max() <= 1e-12
        assert np.abs(got - z['f32%d' % n]).max() <= 1e-6
