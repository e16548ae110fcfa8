"""Shared, cached builds of the benchmark pipelines for the tests."""

import functools

from polymage_b200.apps.harris import build_harris
from polymage_b200.apps.unsharp_mask import build_unsharp


@functools.lru_cache(maxsize=None)
def harris(tile=(32, 128)):
    return build_harris(tile_sizes=tile).build()


@functools.lru_cache(maxsize=None)
def unsharp(tile=(32, 128)):
    return build_unsharp(tile_sizes=tile).build()
