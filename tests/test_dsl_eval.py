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
