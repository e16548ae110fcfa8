"""A small mixed request stream (Harris, unsharp mask, 8-level pyramid
blending on uneven sizes) served in batches under a tight memory budget,
so that it is cut into several chunks; every request's output is checked
against the oracle with the single-image tolerances (Harris 1e-5
relative, unsharp 1e-5 where the select margin exceeds 1e-6, pyramid
2e-5)."""

import numpy as np
import pytest

import oracle.harris as OH
import oracle.pyramid as OP
import oracle.unsharp as OU
from polymage_b200.apps import stream

pytestmark = pytest.mark.gpu


def test_mixed_stream_matches_oracle(cuda):
    reqs = stream.make_stream(12, seed=3, lo=256, hi=640)
    assert len(set(k for k, _, _ in reqs)) == 3
    r = stream.serve(reqs, device=cuda, budget=24 << 20, seed=3, keep=True)
    assert r["chunks"] > 1
    for kind, prm, ins, outs in r["requests"]:
        if kind == 'harris':
            img = ins['img'].cpu().numpy()
            ref = OH.harris(img)
            got = outs['harris'].cpu().numpy()
            # written: [2, rows-3] x [2, cols-3] (the outputs start
            # uninitialized, so only written points are compared)
            inner = (slice(2, img.shape[0] - 2), slice(2, img.shape[1] - 2))
            err = np.abs(got[inner] - ref[inner]).max() / np.abs(ref).max()
            assert err <= 1e-5, err
        elif kind == 'unsharp':
            img = ins['img'].cpu().numpy()
            ref = OU.unsharp(img, 0.001, 3.0)
            ok = OU.margin(img, 0.001) > 1e-6
            R, C = prm['R'], prm['C']
            ok[:, R - 1, :] = False            # never written
            ok[:, :, C - 1] = False
            d = np.abs(outs['mask'].cpu().numpy().astype(np.float64) - ref)
            assert d[ok].max() <= 1e-5, d[ok].max()
        else:
            ref = OP.pyramid_blend_clamped(ins['img1'].cpu().numpy(),
                                           ins['img2'].cpu().numpy(),
                                           ins['mask'].cpu().numpy(), L=8)
            err = np.abs(outs['blend'].cpu().numpy().astype(np.float64) -
                         ref).max()
            assert err <= 2e-5, err
