"""The pipelines this backend ships prebuilt, with their default (tuned)
settings."""

import functools

from .harris import build_harris
from .unsharp_mask import build_unsharp


def default_builds():
    return [
        ("harris", functools.partial(build_harris, tile_sizes=(32, 128))),
        ("unsharp", functools.partial(build_unsharp, tile_sizes=(32, 128))),
    ]
