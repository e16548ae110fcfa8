"""Compiler entry point (sandbox/compiler.py:33-80).

``buildPipeline`` keeps the reference's keyword arguments and defaults:
``group_size`` 5, ``tile_sizes`` [16, 16, 16], ``size_threshold`` 200*200,
and ``optimize_storage`` implying ``flatten_scratchpad``.  The reference's
C-target options (``early_free``, ``pool_alloc``, ``multipar``) are
accepted and have no effect.  Options may also carry CUDA-target settings
as ``"name=value"`` strings or ``(name, value)`` tuples:

* kernel shape: ``threads`` (CTA size), ``rblock=K`` (rows per thread on
  interior tiles), ``min_blocks=N`` (resident CTAs per SM asked of ptxas),
  ``tile`` (tile sizes overriding ``tile_sizes``), ``red_tile`` (tile of
  a Reduction's domain);
* fusion and storage: ``inline_budget`` (register-recompute budget per
  consumer point), ``smem_budget`` (bytes per CTA), ``materialize`` (names
  kept in shared memory), ``no_stage`` (never stage inputs in shared
  memory), ``tight_stage`` (no TMA slack for narrow whole innermost
  dimensions), ``no_privatize`` (reductions accumulate straight into
  HBM), ``no_storage_reuse``;
* expressions: ``separable`` (rank-one rectangular weighted sums of one
  producer, at least six terms, summed as row sums: polymage_b200/
  separable.py);
* grouping beyond the reference's: ``fuse_all`` (every non-const stage in
  one group when legal), ``('merge_small', N)`` (a group merges into its
  only child when both have stages of at most N points);
* staging and tiling: ``stage_pointwise`` (inputs read at one offset are
  staged too), ``prefetch`` (a CTA loads its next tile while computing
  this one), ``channel_tile`` (a small leading channel dimension tiled
  whole), ``oob_zero`` (reads outside a producer's domain read 0),
  ``no_row_pad``, ``no_tile_shrink``, ``('storage_order', ((name,
  dims), ...))`` (an intermediate array's dimensions, outermost to
  innermost in memory);
* reductions: ``red_unroll=N``, ``red_spread``, ``no_gather`` (scatter
  form instead of output-stationary);
* launches: ``streams=N`` (concurrent streams for independent groups, 1
  for the caller's stream only), ``pdl`` (programmatic stream
  serialization), ``chain`` / ``('chain', N)`` (consecutive stencil groups
  of at most N tiles each as phases of one launch, grid barriers between
  dependent phases);
* switches of single optimisations, for measurement and debugging:
  ``shared_regions`` (one thread computes a tile's regions and shares
  them through shared memory), ``no_inside`` (every tile on the general
  path), ``guarded`` (one point per iteration), ``no_vec``, ``no_vec2``,
  ``no_cblock``, ``no_static_res``, ``no_fold_clamps``.
"""

from .pipe import Pipeline


def buildPipeline(outputs,
                  param_estimates=[],
                  param_constraints=[],
                  grouping=[],
                  group_size=None,
                  inline_directives=[],
                  tile_sizes=[],
                  size_threshold=None,
                  pipe_name=None,
                  options=[]):
    outputs = list(dict.fromkeys(outputs))
    if group_size is None:
        group_size = 5
    if not tile_sizes:
        tile_sizes = [16, 16, 16]
    if size_threshold is None:
        size_threshold = 200 * 200
    options = list(options)
    if 'optimize_storage' in options and 'flatten_scratchpad' not in options:
        options.append('flatten_scratchpad')
    return Pipeline(_outputs=outputs,
                    _param_estimates=param_estimates,
                    _param_constraints=param_constraints,
                    _grouping=grouping,
                    _group_size=group_size,
                    _inline_directives=inline_directives,
                    _tile_sizes=tile_sizes,
                    _size_threshold=size_threshold,
                    _name=pipe_name,
                    _options=options)
