"""DSL definitions evaluated point by point (tests/dsl_eval.py, FP64, no
compiler involved) against the oracles: checks the pipeline statements
themselves.  The local Laplacian statement reproduces the reference's own
compiled output exactly; the interpolation restatement (parity unpinned:
no reference output exists for it) reproduces its DSL statement."""

import os
import sys

import numpy as np

from tests.dsl_eval import Evaluator

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.setrecursionlimit(max(sys.getrecursionlimit(), 20000))


def test_evaluator_matches_pinned_harris_oracle():
    import oracle.harris as OH
    from polymage_b200.apps.harris import harris_pipe
    img = OH.make_input(20, 24, seed=1)
    ev = Evaluator({'R': 18, 'C': 22}, {'img': img.astype(np.float64)})
    got = ev.array(harris_pipe({}))
    ref = OH.harris(img)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_local_laplacian_statement_reproduces_reference_output():
    from polymage_b200.apps.local_laplacian import local_laplacian
    z = np.load(os.path.join(GOLD, "laplacian.npz"))
    f = z['frame0']
    ev = Evaluator({'R': f.shape[0] + 92, 'C': f.shape[1] + 92,
                    'alpha': float(z['alpha']), 'beta': float(z['beta'])},
                   {'img_colour': f})
    got = ev.array(local_laplacian({}))
    assert np.array_equal(got, z['out0'].astype(np.float64))


def test_interpolate_restatement_matches_statement():
    import oracle.interpolate as OI
    from polymage_b200.apps.interpolate import interpolate
    for R, C in ((16, 16), (21, 13)):
        img = OI.make_input(R, C, seed=R)
        ev = Evaluator({'R': R, 'C': C}, {'img': img.astype(np.float64)})
        got = ev.array(interpolate({}))
        assert np.abs(got - OI.interpolate(img)).max() <= 1e-12


def test_unsharp_statement_matches_pinned_oracle():
    import oracle.unsharp as OU
    from polymage_b200.apps.unsharp_mask import unsharp_mask
    R, C = 12, 17
    img = OU.make_input(R, C, seed=3)
    ev = Evaluator({'R': R, 'C': C, 'threshold': 0.001, 'weight': 3.0},
                   {'img': img.astype(np.float64)})
    got = ev.array(unsharp_mask({}))
    ok = OU.margin(img, 0.001) > 1e-6
    assert np.abs(got - OU.unsharp(img, 0.001, 3.0))[ok].max() <= 1e-12


def test_pyramid_statements_match_oracles():
    import oracle.pyramid as OP
    from polymage_b200.apps.pyramid_blend import (pyramid_blending,
                                                  pyramid_blending_clamped)
    R, C = 96, 100
    i1, i2, m = OP.make_inputs(R, C, seed=1)
    imgs = {'img1': i1.astype(np.float64), 'img2': i2.astype(np.float64),
            'mask': m.astype(np.float64)}
    got = Evaluator({'R': R, 'C': C}, imgs).array(pyramid_blending({}))
    assert np.abs(got - OP.pyramid_blend(i1, i2, m)).max() <= 1e-12
    R, C = 37, 53
    i1, i2, m = OP.make_inputs(R, C, seed=2)
    imgs = {'img1': i1.astype(np.float64), 'img2': i2.astype(np.float64),
            'mask': m.astype(np.float64)}
    got = Evaluator({'R': R, 'C': C}, imgs).array(
        pyramid_blending_clamped({}, L=8))
    ref = OP.pyramid_blend_clamped(i1, i2, m, L=8)
    assert np.abs(got - ref).max() <= 1e-12


def test_bilateral_statement_matches_oracle():
    """The grid is a Reduction: accumulated sequentially over the image;
    the oracle bins z in float32 (as the kernel does), the evaluator in
    FP64, hence the tolerance."""
    import oracle.bilateral as OB
    from polymage_b200.apps.bilateral_grid import bilateral_grid
    rows, cols = 40, 48
    img = OB.make_input(rows, cols, seed=5)
    got = Evaluator({'rows': rows, 'cols': cols},
                    {'input': img.astype(np.float64)}).array(
        bilateral_grid({}))
    assert np.abs(got - OB.bilateral(img)).max() <= 1e-6


def test_campipe_statement_matches_c_restatement():
    """Integer pipeline; the evaluator computes the const LUT in FP64 where
    the restatement uses the reference's float/double mix, so an entry may
    round differently: at most one count on at most 1 % of the bytes."""
    import oracle.campipe as OC
    from polymage_b200.apps.campipe import (camera_pipe, MATRIX_3200,
                                            MATRIX_7000)
    R, C = 80, 96
    img = OC.make_input(R, C, seed=4)
    ev = Evaluator({'R': R, 'C': C, 'colour_temp': 3700.0, 'contrast': 50.0,
                    'gamma': 2.0},
                   {'img': img.astype(np.int64),
                    'matrix_3200': np.array(MATRIX_3200),
                    'matrix_7000': np.array(MATRIX_7000)})
    got = ev.array(camera_pipe({}))
    d = np.abs(got - OC.campipe(img, 3700.0, 50.0, 2.0).astype(np.float64))
    assert d.max() <= 1 and (d > 0).mean() <= 0.01


def test_jacobi_restatement_matches_statement():
    import oracle.jacobi as OJ
    from polymage_b200.apps.jacobi import jacobi2d
    for N, T in ((10, 1), (13, 4)):
        V, F = OJ.make_input(N, seed=N)
        got = Evaluator({'N': N}, {'V_': V, 'F_': F}).array(
            jacobi2d({}, T=T))
        assert np.abs(got - OJ.jacobi2d(V, F, T)).max() <= 1e-12


def test_jacobi3d_restatement_matches_statement():
    import oracle.jacobi as OJ
    from polymage_b200.apps.jacobi import jacobi3d
    N, T = 6, 2
    rng = np.random.default_rng(1)
    V, F = rng.random((N + 2,) * 3), rng.random((N + 2,) * 3)
    got = Evaluator({'N': N}, {'V_': V, 'F_': F}).array(jacobi3d({}, T=T))
    assert np.abs(got - OJ.jacobi3d(V, F, T)).max() <= 1e-12


def test_v_cycle_restatement_matches_statement():
    import oracle.multigrid as OM
    from polymage_b200.apps.multigrid import v_cycle
    for n, L, g in ((3, 2, 1), (4, 1, 1), (2, 3, 1), (3, 2, 2), (2, 3, 2)):
        V, F = OM.make_input(n, L, seed=n)
        got = Evaluator({'n': n}, {'V_': V, 'F_': F}).array(
            v_cycle({}, L=L, gamma=g, name="Wcycle" if g == 2 else "Vcycle"))
        assert np.abs(got - OM.v_cycle(V, F, n, L, gamma=g)).max() <= 1e-12


def test_v_cycle3d_restatement_matches_statement():
    import oracle.multigrid as OM
    from polymage_b200.apps.multigrid import v_cycle
    for n, L, g in ((1, 2, 1), (2, 1, 1), (1, 2, 2)):
        V, F = OM.make_input3d(n, L, seed=n)
        got = Evaluator({'n': n}, {'V_': V, 'F_': F}).array(
            v_cycle({}, L=L, gamma=g, dims=3))
        assert np.abs(got - OM.v_cycle3d(V, F, n, L, gamma=g)).max() <= 1e-12


def test_nas_mg_restatement_matches_statement():
    """Both outputs of the NAS MG V-cycle (MG_U, MG_R)."""
    import oracle.nas_mg as ON
    from polymage_b200.apps.nas_mg import mg3p
    for n in (8, 16):
        U, V, R = ON.make_input(n, seed=n)
        u, r = mg3p({}, lt=n.bit_length() - 1, prob_class='S')
        ev = Evaluator({'n': n}, {'U': U, 'V': V, 'R': R})
        ou, orr = ON.mg3p(U, V, R, 'S')
        assert np.abs(ev.array(u) - ou).max() <= 1e-12
        assert np.abs(ev.array(r) - orr).max() <= 1e-12


def test_nlmeans_restatement_matches_statement():
    """Non-local means (image channel 3 read as 0, option 'oob_zero')."""
    import oracle.nlmeans as ONL
    from polymage_b200.apps.nlmeans import nlmeans
    R, C, p, s = 13, 15, 3, 3
    img = ONL.make_input(R, C, seed=1)
    ev = Evaluator({'R': R, 'C': C, 'patch_size': p, 'search_area': s},
                   {'img': img.astype(np.float64)}, oob_zero=True)
    got = ev.array(nlmeans({}))
    assert np.abs(got - ONL.nlmeans(img, p, s)).max() <= 1e-12


def test_maxfilter_restatement_matches_statement():
    """Max filter (vert_log read as 0 outside its domain, option
    'oob_zero'; data-dependent slice indices clamped)."""
    import oracle.maxfilter as OMF
    from polymage_b200.apps.max_filter import maxfilter
    R, C = 84, 196
    img = OMF.make_input(R, C, seed=2)
    ev = Evaluator({'R': R, 'C': C}, {'img': img.astype(np.float64)},
                   oob_zero=True)
    got = ev.array(maxfilter({}))
    ref = OMF.maxfilter(img)
    assert (ref > 0).any() and np.array_equal(got, ref)
