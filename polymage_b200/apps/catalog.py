"""The pipelines this backend ships prebuilt, with their default settings
(tile sizes and register blocking chosen by measurement on B200)."""

import functools

from .harris import build_harris
from .unsharp_mask import build_unsharp

HARRIS = dict(tile_sizes=(32, 64), options=('rblock=4',))
UNSHARP = dict(tile_sizes=(32, 128), options=('rblock=8',))


def default_builds():
    return [
        ("harris", functools.partial(build_harris, **HARRIS)),
        ("unsharp", functools.partial(build_unsharp, **UNSHARP)),
    ]
