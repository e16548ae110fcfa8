"""Shared, cached builds of the benchmark pipelines for the tests."""

import functools

from polymage_b200.apps import catalog
from polymage_b200.apps.harris import build_harris
from polymage_b200.apps.unsharp_mask import build_unsharp


@functools.lru_cache(maxsize=None)
def harris(tile=None):
    if tile is None:
        return build_harris(**catalog.HARRIS).build()
    return build_harris(tile_sizes=tile).build()


@functools.lru_cache(maxsize=None)
def unsharp(tile=None):
    if tile is None:
        return build_unsharp(**catalog.UNSHARP).build()
    return build_unsharp(tile_sizes=tile).build()
