"""The pipelines this backend ships prebuilt, with their default settings:
the best of exhaustive tuning on B200 at each pipeline's benchmark size
(15 tile shapes x 5 group sizes x register blocking 2/4/8, min of five
timed runs each with L2 flushed; polymage_b200.autotune).  Harris keeps the
group size of the reference's Harris builder (11: all stages in one group,
harris/builder.py:66-67), which is outside the tuned group sizes (3..10)
and faster than their best (0.029 vs 0.034 ms).  Unsharp recomputes blurx
inside blury (a larger inline budget), also outside the tuned space: with
16-byte shared-memory reads the recomputation is cheaper than a second
shared-memory stage and its barrier (0.087-0.090 vs 0.094 ms for the
tuned best); CTAs of 128 threads on 64x128 tiles with 16 rows per thread
keep more, smaller CTAs resident (0.0773 vs 0.0866 ms with 256 threads).
Harris also runs 128-thread CTAs, on 32x64 tiles (0.0273 vs 0.0291 ms).
The bilateral grid's construction takes 16x256-pixel tiles (0.0908 vs
0.1033 ms with 32x256), and its slicing group stages the input pixels by
TMA although it reads each once (option stage_pointwise: 0.0728 vs 0.0786
ms; the same option slows the pyramids and the local Laplacian), interpolation 32x64 tiles (0.53 vs 1.69 ms with
the reference builder's 16x16).  The camera pipe fuses every stage into one
group (option fuse_all; the greedy grouping leaves six kernels: 0.133 vs
0.190 ms) and tiles its three output channels whole (option channel_tile:
a thread computes a pixel's red, green and blue once for all three
channels, 0.085 vs 0.130 ms) on 32x128 tiles with 4 rows per thread.
Harris and both pyramids ask ptxas for 4 resident CTAs per SM
(``min_blocks=4``: at most 64 registers a thread), also outside the tuned
space: 0.0290 vs 0.0303 ms, 0.203 vs 0.209 ms and
0.218 vs 0.227 ms (the 8-level pyramid with its interior tiles reading
clamped taps unclamped); the bilateral grid is slower with it (0.108 vs
0.107 ms) and unsharp is bound by shared memory, not registers.
The widening pipelines' settings are the best of smaller sweeps
(polymage_b200.apps.measure, same timing): Jacobi 2-D 32x64 tiles with 5
steps per group (0.133 vs 0.207 ms for 16x64 with 10), Jacobi 3-D and the
3-D multigrid cycles unfused (group size 1) on 8x16x32 and 8x16x64 tiles
(0.164 vs 0.356 ms; 3.2 vs 8.6 ms): in 3-D the halo of a fused time step
grows every face of a tile, so recomputation costs more than the HBM
round trip it saves.  The Jacobi steps, the 2-D multigrid cycles and NAS MG
also stage their pointwise-read right-hand sides by TMA (option
stage_pointwise: Jacobi 2-D 0.116 vs 0.132 ms, 3-D 0.154 vs 0.165 ms,
V-cycle 0.073 vs 0.083 ms, W-cycle 0.138 vs 0.155 ms, NAS MG 0.255 vs
0.264 ms; the 3-D cycles are slower with it).
A later sweep of the CTA-shape knobs (same timing, one box): the camera
pipe with 3 resident CTAs asked of ptxas (0.0491 vs 0.0553 ms), the L=4
pyramid with 4 rows per thread and its tile regions computed by one
thread (option shared_regions: 0.1735 vs 0.1875 ms; every other pipeline
is slower with that option), the L=8 pyramid and the local Laplacian with
4 rows per thread (0.2164 vs 0.2237 ms, 0.1474 vs 0.1496 ms),
interpolation with 3 resident CTAs (0.3048 vs 0.3138 ms).  Harris sums
its 3x3 box sums and Sobel taps as row sums that the rows of a thread's
block share (option separable: 0.0255 vs 0.0274 ms).  The 2-D multigrid
cycles take 8x32 tiles: their 255^2 grids give 16x64 tiles too few CTAs
for 148 SMs (V-cycle 0.061 vs 0.075 ms, W-cycle 0.113 vs 0.140 ms)."""

import functools

from .harris import build_harris
from .unsharp_mask import build_unsharp
from .campipe import build_campipe
from .bilateral_grid import build_bilateral
from .pyramid_blend import build_pyramid, build_pyramid_clamped
from .local_laplacian import build_laplacian
from .interpolate import build_interpolate
from .jacobi import build_jacobi2d, build_jacobi3d
from .multigrid import build_v_cycle
from .nas_mg import build_mg3p
from .nlmeans import build_nlmeans
from .max_filter import build_maxfilter

HARRIS = dict(tile_sizes=(32, 64), group_size=11,
              options=('rblock=8', 'min_blocks=4', 'threads=128',
                       'separable'))
UNSHARP = dict(tile_sizes=(64, 128), group_size=10,
               options=('rblock=16', 'inline_budget=400', 'threads=128'))
CAMPIPE = dict(tile_sizes=(32, 128), group_size=12,
               options=('rblock=4', 'fuse_all', 'channel_tile',
                        'min_blocks=3'))
BILATERAL = dict(tile_sizes=(1, 32, 128), group_size=10,
                 options=(('red_tile', (16, 256)), 'rblock=4',
                          'stage_pointwise'))
PYRAMID = dict(tile_sizes=(32, 64), group_size=10,
               options=('rblock=4', 'min_blocks=4', 'shared_regions'))
# 8 levels, indices clamped at every level's borders (any image size)
PYRAMID8 = dict(L=8, tile_sizes=(32, 64), group_size=10,
                options=('rblock=4', 'min_blocks=4'))

# local Laplacian filter (the video demo's pipeline_laplacian), 1080p frames
# (option tight_stage: the uint8 [x][y][3] frame is staged without the TMA
# alignment slack of its 3-byte innermost rows, 0.148 vs 0.213 ms)
LAPLACIAN = dict(tile_sizes=(32, 64), group_size=10,
                 options=('rblock=4', 'tight_stage'))

# The widening pipelines at the reference Makefiles' settings: Jacobi 2-D
# N=2048 and 3-D N=128 with 10 steps each (stencil/jacobi{2D,3D}/
# Makefile:10-11), multigrid cycles with L=3 levels above a 31-point coarse
# grid, 10 pre-smoothings and none after or on the coarsest level
# (multigrid/jacobi{2D,3D}/Makefile:10-16), NAS MG class W (NAS-PB-MG-3.2/
# Makefile:9), interpolation of a 2048x2048 RGBA image.
INTERPOLATE = dict(rows=2048, cols=2048, tile_sizes=(32, 64), group_size=11,
                   options=('min_blocks=3',))
JACOBI2D = dict(N=2048, T=10, tile_sizes=(32, 64), group_size=5,
                options=('stage_pointwise',))
JACOBI3D = dict(N=128, T=10, tile_sizes=(8, 16, 32), group_size=1,
                options=('stage_pointwise',))
VCYCLE = dict(n=31, L=3, nu1=10, nu2=0, nuc=0, tile_sizes=(8, 32),
              group_size=6, options=('stage_pointwise',))
WCYCLE = dict(VCYCLE, gamma=2, name="Wcycle")
VCYCLE3D = dict(n=31, L=3, nu1=10, nu2=0, nuc=0, dims=3,
                tile_sizes=(8, 16, 64), group_size=1, name="Vcycle3d")
WCYCLE3D = dict(VCYCLE3D, gamma=2, name="Wcycle3d")
MG3P = dict(prob_class='W', tile_sizes=(4, 8, 32), group_size=6,
            options=('stage_pointwise',))
# non-local means at the reference Makefile's patch size and search area
# (non_local_means/Makefile:11-12) on a 256x256 image
NLMEANS = dict(rows=256, cols=256)
# max filter (radius 26) on a 1536x2560 landscape image: the spec's
# vert_log rows are [26, C-R-79], non-empty only when C > R + 104
# (tiles of 8 x 32 pixels x 3 channels for its reductions)
# (its vert_log and vert arrays are stored slice-outermost, so that the
# final maximum's gather, whose warp spans channels and columns at one
# slice, reads contiguous words: 1.137 vs 1.388 ms)
MAXFILTER = dict(rows=1536, cols=2560,
                 options=('oob_zero', ('red_tile', (8, 32, 3, 16)),
                          ('storage_order', (('vert', (3, 0, 1, 2)),
                                             ('vert_log', (3, 0, 1, 2))))))

_BUILDERS = {
    "harris": (build_harris, HARRIS),
    "unsharp": (build_unsharp, UNSHARP),
    "campipe": (build_campipe, CAMPIPE),
    "bilateral": (build_bilateral, BILATERAL),
    "pyramid": (build_pyramid, PYRAMID),
    "pyramid8": (build_pyramid_clamped, PYRAMID8),
    "laplacian": (build_laplacian, LAPLACIAN),
    "interpolate": (build_interpolate, INTERPOLATE),
    "jacobi2d": (build_jacobi2d, JACOBI2D),
    "jacobi3d": (build_jacobi3d, JACOBI3D),
    "vcycle": (build_v_cycle, VCYCLE),
    "wcycle": (build_v_cycle, WCYCLE),
    "vcycle3d": (build_v_cycle, VCYCLE3D),
    "wcycle3d": (build_v_cycle, WCYCLE3D),
    "mg3p": (build_mg3p, MG3P),
    "nlmeans": (build_nlmeans, NLMEANS),
    "maxfilter": (build_maxfilter, MAXFILTER),
}

_cache = {}


def default_builds():
    return [(name, functools.partial(b, **kw))
            for name, (b, kw) in _BUILDERS.items()]


def build(name):
    """The compiled default build of a shipped pipeline (cached)."""
    if name not in _cache:
        b, kw = _BUILDERS[name]
        _cache[name] = b(**kw).build()
    return _cache[name]


def variant(name, extra_options=(), drop_options=()):
    """The uncompiled pipeline of a shipped build with options added
    (``extra_options``) or removed (``drop_options``)."""
    import inspect
    b, kw = _BUILDERS[name]
    kw = dict(kw)
    base = kw.get('options')
    if base is None:
        base = inspect.signature(b).parameters['options'].default
    opts = [o for o in base if o not in drop_options]
    kw['options'] = tuple(opts) + tuple(extra_options)
    return b(**kw)
