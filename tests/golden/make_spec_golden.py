"""Regenerate the fixtures that pin the restatements of the pipelines the
reference ships no generated code for, from the reference's own DSL specs
(loaded unmodified from the reference tree and evaluated point by point
by tests/golden/refspec.py):

  python tests/golden/make_spec_golden.py      (a few minutes)

campipe_spec.npz    camera_pipe (sandbox/apps/python/img_proc/campipe/
                    polymage_campipe.py:13-304) with C semantics: output
                    ``process`` for a 64x96 raw (seed 5; colour_temp 3700,
                    contrast 50, gamma 2) and a 70x101 raw (seed 6; 5000,
                    40, 1.8), plus the const functions ``matrix`` and the
                    whole ``curveLUT`` (v = -32768..32767) of the first set
bilateral_spec.npz  bilateral_grid (bilateral_grid/polymage_bilateral_grid.
                    py:16-130) on 40x56 (seed 40) and 37x61 (seed 37)
                    float32 images: ``filtered`` in FP64 (z bins as the
                    compiled code takes them) and with the compiled code's
                    float arithmetic
pyramid_spec.npz    pyramid_blending (pyramid_blend/polymage_blending.py:
                    13-196, L = 4) on 96x100 (seed 96) and 101x117 (seed
                    101) inputs: ``blend`` over its domain box, in FP64 and
                    with float arithmetic, and the box's lower corner

Inputs come from the oracle's own ``make_input(s)`` so the fixtures hold
exactly what the tests feed the restatements.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.setrecursionlimit(max(sys.getrecursionlimit(), 50000))

from tests.golden import refspec as RS  # noqa: E402
import oracle.bilateral as OB  # noqa: E402
import oracle.campipe as OC  # noqa: E402
import oracle.pyramid as OP  # noqa: E402

CAMPIPE_CASES = ((64, 96, 5, 3700.0, 50.0, 2.0),
                 (70, 101, 6, 5000.0, 40.0, 1.8))
BILATERAL_CASES = ((40, 56), (37, 61))
PYRAMID_CASES = ((96, 100), (101, 117))


def campipe():
    mod = RS.load_spec("campipe", "polymage_campipe.py")
    arrs = {}
    for n, (R, C, seed, kelvin, contrast, gamma) in enumerate(CAMPIPE_CASES):
        out = mod.camera_pipe({})
        img = OC.make_input(R, C, seed=seed)
        ev = RS.CEvaluator({'R': R, 'C': C, 'colour_temp': kelvin,
                            'contrast': contrast, 'gamma': gamma},
                           {'img': img, 'matrix_3200': OC.MATRIX_3200,
                            'matrix_7000': OC.MATRIX_7000})
        arrs['img%d' % n] = img
        arrs['params%d' % n] = np.array([kelvin, contrast, gamma],
                                        np.float32)
        arrs['out%d' % n], _ = ev.array(out)
        if n == 0:
            arrs['matrix'], _ = ev.array(ev.function_named(out, 'matrix'))
            arrs['lut'], _ = ev.array(ev.function_named(out, 'curveLUT'))
    np.savez_compressed(os.path.join(HERE, "campipe_spec.npz"), **arrs)


def bilateral():
    mod = RS.load_spec("bilateral_grid", "polymage_bilateral_grid.py")
    arrs = {}
    for n, (rows, cols) in enumerate(BILATERAL_CASES):
        img = OB.make_input(rows, cols, seed=rows)
        arrs['img%d' % n] = img
        for tag, fp64 in (('fp64', True), ('f32', False)):
            ev = RS.CEvaluator({'rows': rows, 'cols': cols}, {'input': img},
                               fp64=fp64)
            arrs['%s%d' % (tag, n)], _ = ev.array(mod.bilateral_grid({}))
    np.savez_compressed(os.path.join(HERE, "bilateral_spec.npz"), **arrs)


def pyramid():
    mod = RS.load_spec("pyramid_blend", "polymage_blending.py")
    arrs = {}
    for n, (R, C) in enumerate(PYRAMID_CASES):
        i1, i2, m = OP.make_inputs(R, C, seed=R)
        arrs['shape%d' % n] = np.array([R, C])
        for tag, fp64 in (('fp64', True), ('f32', False)):
            ev = RS.CEvaluator({'R': R, 'C': C},
                               {'img1': i1, 'img2': i2, 'mask': m},
                               fp64=fp64)
            arrs['%s%d' % (tag, n)], lo = ev.array(mod.pyramid_blending({}))
        arrs['lo%d' % n] = np.array(lo)
    np.savez_compressed(os.path.join(HERE, "pyramid_spec.npz"), **arrs)


def main():
    campipe()
    bilateral()
    pyramid()
    print("wrote campipe_spec.npz, bilateral_spec.npz, pyramid_spec.npz")


if __name__ == "__main__":
    main()
