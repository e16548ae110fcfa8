"""Regenerate the golden fixtures from the reference's own generated C++
(oracle/_ref, built by `make -C oracle` from the reference tree).

  python tests/golden/make_golden.py

harris.npz   refHarris (sandbox/ipp_bench/harris/harris_function.cpp) on a
             40x56 float32 image, U[0,1) seed 123
unsharp.npz  pipeline_mask (sandbox/video_demo/unsharp_polymage.cpp) on a
             (24+4)x(37+4)x3 uint8 image, seed 321, threshold 0.001, w 3
laplacian.npz  pipeline_laplacian (sandbox/video_demo/laplacian_
             polymage.cpp) on 64x96x3 and 75x131x3 uint8 frames, seeds 7
             and 8, alpha 1/3, beta 1 (the video demo's settings)
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle.ref as ref  # noqa: E402


def main():
    rng = np.random.default_rng(123)
    img = rng.random((40, 56), dtype=np.float32)
    np.savez_compressed(os.path.join(HERE, "harris.npz"), img=img,
                        out=ref.ref_harris(img))
    rng = np.random.default_rng(321)
    u8 = rng.integers(0, 256, (24 + 4, 37 + 4, 3), dtype=np.uint8)
    out = ref.ref_unsharp(u8, 0.001, 3.0)
    np.savez_compressed(os.path.join(HERE, "unsharp.npz"), img=u8, out=out,
                        threshold=np.float32(0.001), weight=np.float32(3.0))
    arrs = {}
    for n, (seed, h, w) in enumerate(((7, 64, 96), (8, 75, 131))):
        frame = np.random.default_rng(seed).integers(0, 256, (h, w, 3),
                                                     dtype=np.uint8)
        arrs['frame%d' % n] = frame
        arrs['out%d' % n] = ref.ref_laplacian(frame, 1.0 / 3.0, 1.0)
    np.savez_compressed(os.path.join(HERE, "laplacian.npz"),
                        alpha=np.float32(1.0 / 3.0), beta=np.float32(1.0),
                        **arrs)
    print("wrote harris.npz, unsharp.npz, laplacian.npz")


if __name__ == "__main__":
    main()
