"""Compiler passes and plans (no GPU): grouping, materialization,
static extents vs exhaustive region simulation, validation and codegen."""

import numpy as np
import pytest

from polymage_b200.constructs import *   # noqa: F401,F403
from polymage_b200.compiler import buildPipeline
from polymage_b200.apps.harris import build_harris
from polymage_b200.apps.unsharp_mask import build_unsharp
from polymage_b200.tiling import infer_regions, PlanError


def test_harris_single_group_like_reference():
    p = build_harris(tile_sizes=(32, 128))
    assert len(p.groups) == 1           # all 11 stages, group_size 11
    plan = p.groups[0].plan
    mat = sorted(f.name for f in plan.steps)
    assert mat == ['Ix', 'Iy', 'harris']
    staged = [n.name for n in plan.nodes if n.role == 'stage']
    assert staged == ['img']
    ext = dict((n.name, n.ext) for n in plan.nodes)
    assert ext['Ix'] == [34, 130] and ext['img'] == [36, 132]


def test_unsharp_plan():
    p = build_unsharp(tile_sizes=(32, 128))
    assert len(p.groups) == 1
    plan = p.groups[0].plan
    assert [f.name for f in plan.steps] == ['blurx', 'mask']
    ext = dict((n.name, n.ext) for n in plan.nodes)
    assert ext['blurx'] == [1, 32, 132] and ext['img'] == [1, 36, 132]
    assert plan.smem_bytes <= 48 * 1024


@pytest.mark.parametrize("build", [build_harris, build_unsharp])
def test_static_extents_bound_every_tile(build):
    """Run region inference for every tile of a small image and check each
    region fits the static (shared-memory) extents."""
    p = build(tile_sizes=(16, 32))
    plan = p.groups[0].plan
    env = p.int_env()
    for k in list(env):
        env[k] = 61 if k.name in ('R', 'C') else env[k]
    anchor = plan.anchor
    dom = [(int(__import__('polymage_b200.evaluate', fromlist=['x'])
                .eval_int(d.lowerBound, env)),
            int(__import__('polymage_b200.evaluate', fromlist=['x'])
                .eval_int(d.upperBound, env))) for d in anchor.domain]
    T = plan.tile
    starts = [range(lo, hi + 1, t) for (lo, hi), t in zip(dom, T)]
    import itertools
    for origin in itertools.product(*starts):
        box = [(o, min(o + t - 1, hi)) for o, t, (lo, hi) in
               zip(origin, T, dom)]
        regs = infer_regions(plan, box, env)
        for n in plan.nodes:
            if n.role in ('global', 'inline'):
                continue
            lo, hi = regs[n.func]
            for d in range(n.ndims):
                assert int(hi[d]) - int(lo[d]) + 1 <= n.ext[d]


def test_out_of_domain_reference_rejected():
    R = Parameter(Int, "R")
    x = Variable(Int, "x")
    img = Image(Float, "img", [R])
    f = Function(([x], [Interval(Int, 0, R - 1)]), Float, "f")
    f.defn = [img(x + 1)]
    with pytest.raises(TypeError):
        buildPipeline([f], param_estimates=[(R, 100)])


def test_inconsistent_scaling_splits_group():
    """A stage read both at x and x/2 cannot be tiled with the reader."""
    R = Parameter(Int, "R")
    x = Variable(Int, "x")
    img = Image(Float, "img", [R])
    a = Function(([x], [Interval(Int, 0, R - 1)]), Float, "a")
    a.defn = [img(x) * 2.0]
    b = Function(([x], [Interval(Int, 0, R - 1)]), Float, "b")
    b.defn = [a(x) + a(x / 2)]
    p = buildPipeline([b], param_estimates=[(R, 4096)], group_size=5)
    assert len(p.groups) == 2


def test_generated_source_has_tma_and_no_multicast():
    p = build_unsharp(tile_sizes=(32, 128))
    src = p.generate_code().source
    assert 'pm_tma_load_3d' in src
    assert 'multicast' not in src
    assert '__launch_bounds__' in src


def test_grouping_respects_group_size():
    p = build_harris(tile_sizes=(32, 128), group_size=3)
    assert all(len(g.comps) <= 3 for g in p.groups)
    assert len(p.groups) > 1


def test_clamped_taps_are_monotone():
    """min/max of indices monotone in the same direction are monotone (the
    clamped taps of the 8-level pyramid)."""
    from polymage_b200.evaluate import is_min_max, monotone_dir
    R = Parameter(Int, "R")
    x = Variable(Int, "x")
    e = Min(Max(2 * x - 2, 0), (R + 63) / 64 - 1)
    assert is_min_max(e)
    assert monotone_dir(e, x) == 1
    assert monotone_dir(Min(Max(7 - x, 0), R - 1), x) == -1
    assert monotone_dir(Max(x, 5 - x), x) is None


def test_level_size_divisions_do_not_enter_the_period():
    """A stage decimating a level whose size is (R + 63) / 64: the tile
    origin period is 1 (the division is of parameters only), and the
    staged producer's static extent covers the clamped 5-tap footprint of
    a 32-row tile (2 * 32 + 3 rows)."""
    from polymage_b200.evaluate import divisors_in
    R = Parameter(Int, "R")
    C = Parameter(Int, "C")
    x = Variable(Int, "x")
    y = Variable(Int, "y")
    n6 = (R + 63) / 64
    n7 = (R + 127) / 128
    img = Image(Float, "img", [R, C])
    a = Function(([x, y], [Interval(Int, 0, n6 - 1), Interval(Int, 0, C - 1)]),
                 Float, "a")
    a.defn = [img(Min(64 * x, R - 1), y) * 0.5]
    b = Function(([x, y], [Interval(Int, 0, n7 - 1), Interval(Int, 0, C - 1)]),
                 Float, "b")
    w = (1, 4, 6, 4, 1)
    b.defn = [sum(w[k] * a(Min(Max(2 * x + k - 2, 0), n6 - 1), y)
                  for k in range(5)) * 0.0625]
    assert divisors_in(Min(Max(2 * x - 2, 0), n6 - 1)) == []
    assert divisors_in(x / 2 + n6) == [2]
    p = buildPipeline([b], param_estimates=[(R, 2048), (C, 2048)],
                      tile_sizes=[32, 64], group_size=2,
                      options=[('materialize', ['a'])])
    assert len(p.groups) == 1
    plan = p.groups[0].plan
    assert plan.period == 1
    ext = dict((n.name, n.ext) for n in plan.nodes)
    assert ext['a'] == [67, 64]


def test_interior_tiles_check_clamps_before_reading_unclamped():
    """A clamped tap is read unclamped on interior tiles only: the
    interior test compares each clamped index with its unclamped form at
    both ends of the consumer's region.  Data-dependent clamps (a LUT
    index) are never dropped."""
    R = Parameter(Int, "R")
    C = Parameter(Int, "C")
    x = Variable(Int, "x")
    y = Variable(Int, "y")
    img = Image(Float, "img", [R, C])
    lut = Image(Float, "lut", [256])
    a = Function(([x, y], [Interval(Int, 0, R - 1), Interval(Int, 0, C - 1)]),
                 Float, "a")
    a.defn = [sum(img(Min(Max(x + k - 1, 0), R - 1), y) for k in range(3))]
    b = Function(([x, y], [Interval(Int, 0, R - 1), Interval(Int, 0, C - 1)]),
                 Float, "b")
    b.defn = [lut(Min(Max(Cast(Int, a(x, y) * 64.0), 0), 255))]
    p = buildPipeline([b], param_estimates=[(R, 1024), (C, 1024)],
                      tile_sizes=[32, 64], group_size=2)
    src = p.generate_code().source
    inside = [ln for ln in src.splitlines() if 'const bool pm_inside' in ln]
    assert inside and all(') == (' in ln for ln in inside)
    fast = src[src.index('if (pm_inside)'):]
    fast = fast[:fast.index('} else {') if '} else {' in fast else None]
    # the image taps read unclamped; the LUT index keeps its clamp
    assert 'sm_img[(qb0 - 1) * ' in fast
    assert '< 255) ?' in fast


def test_interleaved_channels_tiled_whole():
    """An anchor [x][y][c] with 3 interleaved channels gets tiles of
    32 x 64 pixels x all channels, not 1 x 32 x 64 (x, y, c); planar
    [c][x][y] anchors keep one channel per tile."""
    from polymage_b200.apps.local_laplacian import build_laplacian
    p = build_laplacian(rows=270, cols=480)
    tiles = dict((g.plan.anchor.name, g.plan.tile) for g in p.groups
                 if g.plan is not None and hasattr(g.plan, 'anchor'))
    assert tiles['laplacian'] == [32, 64, 3]
    assert tiles['gPyramid_L0'] == [1, 32, 64]
    q = build_unsharp(tile_sizes=(32, 128))
    assert q.groups[0].plan.tile == [1, 32, 128]


def test_interpolate_plans_and_compiles():
    """The 10-level interpolation (next app after the benchmark set)
    plans into fused groups and compiles for sm_100a."""
    from polymage_b200.apps.interpolate import build_interpolate
    p = build_interpolate(rows=512, cols=512)
    assert 5 <= len(p.groups) <= 20
    cp = p.build()
    assert cp.so_path.endswith(".so")


def _tile_boxes(plan, env):
    """Every tile of a group's grid, as the kernel enumerates them: the
    union of its live-outs' domains along the anchor dimensions, cut into
    tiles of the plan's sizes."""
    import itertools
    from polymage_b200.evaluate import eval_int
    na = plan.anchor.ndims
    lo = [None] * na
    hi = [None] * na
    for n in plan.nodes:
        if n.role != 'out':
            continue
        for d, dom in enumerate(n.func.domain):
            k = d if n.func is plan.anchor else n.owned_map[d]
            a, b = eval_int(dom.lowerBound, env), eval_int(dom.upperBound, env)
            lo[k] = a if lo[k] is None else min(lo[k], a)
            hi[k] = b if hi[k] is None else max(hi[k], b)
    starts = [range(lo[k], hi[k] + 1, plan.tile[k]) for k in range(na)]
    for origin in itertools.product(*starts):
        yield [(o, min(o + t - 1, h)) for o, t, h in
               zip(origin, plan.tile, hi)]


@pytest.mark.parametrize("name,sizes", [
    ("pyramid8", (256, 300)), ("pyramid8", (37, 53)),
    ("pyramid", (157, 211)), ("campipe", (200, 264)),
    ("laplacian", (64 + 92, 96 + 92)), ("bilateral", (77, 93)),
    ("campipe+fuse_all", (200, 264)), ("campipe+fuse_all", (131, 197))])
def test_static_extents_cover_every_tile_of_every_group(name, sizes):
    """Region inference for every tile of every fused group of a shipped
    pipeline at a small size: each materialized node's region fits the
    static shared-memory extents the kernel was generated with (a region
    larger than its buffer would read or write out of it).  ``+opt``
    adds a build option to the catalog's."""
    from polymage_b200.apps import catalog
    name, _, extra = name.partition('+')
    b, kw = catalog._BUILDERS[name]
    kw = dict(kw)
    if extra:
        kw['options'] = tuple(kw.get('options', ())) + (extra,)
    p = b(**kw)
    env = p.int_env()
    for k in list(env):
        if k.name in ('R', 'rows'):
            env[k] = sizes[0]
        elif k.name in ('C', 'cols'):
            env[k] = sizes[1]
    checked = 0
    for g in p.groups:
        plan = g.plan
        if getattr(plan, 'kind', None) != 'stencil':
            continue
        for box in _tile_boxes(plan, env):
            regs = infer_regions(plan, box, env)
            for n in plan.nodes:
                if not n.in_smem:
                    continue
                lo, hi = regs[n.func]
                for d in range(n.ndims):
                    ext = int(hi[d]) - int(lo[d]) + 1
                    assert ext <= n.ext[d], (n.name, d, ext, n.ext[d], box)
            checked += 1
    assert checked > 0


def test_pipeline_graph_dot(tmp_path):
    """The stage graph as the reference's tests write it
    (pipeline.pipeline_graph.write(...)): one cluster per group, one node
    per stage, one edge per producer-consumer pair, live-outs bold."""
    p = build_harris(tile_sizes=(32, 128))
    g = p.pipeline_graph
    path = tmp_path / "harris.dot"
    g.write(str(path))
    text = path.read_text()
    assert text.startswith('digraph "harris"')
    assert text.count("subgraph") == len(p.groups) == 1
    nodes = [l for l in text.splitlines() if "shape=box" in l]
    assert len(nodes) == len(p.comps) == 11
    edges = sum(len(c.parents) for c in p.comps)
    assert text.count("->") == edges
    assert '"harris" [shape=box, style="rounded, bold"' in text


def test_jacobi_steps_fuse_into_one_time_tiled_group():
    """Four Jacobi steps (one function each) fuse into one overlapped-tile
    group: the time loop is tiled with the space loops; the kernel
    computes in double precision."""
    from polymage_b200.apps.jacobi import build_jacobi2d
    p = build_jacobi2d(N=1022, T=4)
    assert len(p.groups) == 1 and len(p.groups[0].comps) == 4
    src = p.generate_code().source
    assert "double" in src and "4.0f" not in src
    assert p.build().so_path.endswith(".so")
    from polymage_b200.apps.jacobi import build_jacobi3d
    assert build_jacobi3d(N=126, T=2).build().so_path.endswith(".so")


def test_v_cycle_plans_and_compiles():
    """The multigrid V-cycle (3 levels: smoothing, defect, restriction,
    interpolation with correction) fuses across levels and compiles; its
    entry point keeps the reference's name."""
    from polymage_b200.apps.multigrid import build_v_cycle
    p = build_v_cycle(n=63, L=2)
    assert 2 <= len(p.groups) <= 8
    cp = p.build()
    assert cp.so_path.endswith(".so")
    assert "pipeline_Vcycle(" in p.generate_code().source
    w = build_v_cycle(n=63, L=2, gamma=2, name="Wcycle")
    assert w.build().so_path.endswith(".so")
    d3 = build_v_cycle(n=31, L=2, dims=3, tile_sizes=(4, 8, 32),
                       name="Vcycle3d")
    assert d3.build().so_path.endswith(".so")


def test_nas_mg_plans_and_compiles():
    """NAS MG class S: two live-outs (MG_U, MG_R), restrictions down to
    level 1 then the levels back up fused pairwise; compiles."""
    from polymage_b200.apps.nas_mg import build_mg3p
    p = build_mg3p('S')
    names = [c.func.name for g in p.groups for c in g.comps]
    assert "MG_U" in names and "MG_R" in names
    assert p.build().so_path.endswith(".so")


def _next_app(name):
    if name == "interpolate":
        from polymage_b200.apps.interpolate import build_interpolate
        return build_interpolate(rows=128, cols=160), {'R': 128, 'C': 160}
    if name == "jacobi2d":
        from polymage_b200.apps.jacobi import build_jacobi2d
        return build_jacobi2d(N=200, T=4), {'N': 200}
    if name == "vcycle":
        from polymage_b200.apps.multigrid import build_v_cycle
        return build_v_cycle(n=15, L=2), {'n': 15}
    if name == "wcycle3d":
        from polymage_b200.apps.multigrid import build_v_cycle
        return (build_v_cycle(n=7, L=2, dims=3, gamma=2, name="Wcycle3d",
                              tile_sizes=(4, 8, 32)), {'n': 7})
    if name.startswith("catalog:"):
        # the catalog's builds at sizes the GPU tests run them at
        from polymage_b200.apps import catalog
        app, size = name[len("catalog:"):].split("@")
        b, kw = catalog._BUILDERS[app]
        key = {"interpolate": "R", "mg3p": "n"}.get(app, "N")
        if app.endswith("cycle") or app.endswith("cycle3d"):
            key = "n"
        sizes = {key: int(size)}
        if app in ("interpolate", "nlmeans"):
            sizes = {'R': int(size), 'C': int(size) * 3 // 4 + 1}
        if app == "maxfilter":
            sizes = {'R': int(size), 'C': int(size) * 3}
        return b(**kw), sizes
    from polymage_b200.apps.nas_mg import build_mg3p
    return build_mg3p('S'), {'n': 32}


@pytest.mark.parametrize("name", [
    "interpolate", "jacobi2d", "vcycle", "wcycle3d", "nas_mg",
    "catalog:interpolate@211", "catalog:jacobi2d@333",
    "catalog:jacobi3d@47", "catalog:vcycle@20", "catalog:wcycle@13",
    "catalog:vcycle3d@8", "catalog:wcycle3d@6", "catalog:mg3p@128",
    "catalog:nlmeans@37", "catalog:maxfilter@90"])
def test_static_extents_cover_every_tile_next_apps(name):
    """The same tile-by-tile check for the widening apps, at sizes their
    GPU tests run."""
    p, sizes = _next_app(name)
    env = p.int_env()
    for k in list(env):
        if k.name in sizes:
            env[k] = sizes[k.name]
    checked = 0
    for g in p.groups:
        plan = g.plan
        if getattr(plan, 'kind', None) != 'stencil':
            continue
        for box in _tile_boxes(plan, env):
            regs = infer_regions(plan, box, env)
            for n in plan.nodes:
                if not n.in_smem:
                    continue
                lo, hi = regs[n.func]
                for d in range(n.ndims):
                    ext = int(hi[d]) - int(lo[d]) + 1
                    assert ext <= n.ext[d], (n.name, d, ext, n.ext[d], box)
            checked += 1
    assert checked > 0


def test_tight_staging_of_interleaved_channels():
    """Option 'tight_stage': the local Laplacian's uint8 [x][y][3] frame is
    staged with rows of 3 bytes (no TMA slack): the cooperative load loop
    covers 32 x 64 x 3 bytes instead of 32 x 64 x 32, the origin offset is
    0, and the default layout is unchanged."""
    import re
    from polymage_b200.apps.local_laplacian import build_laplacian
    loops = {}
    for opts in (('rblock=8',), ('rblock=8', 'tight_stage')):
        p = build_laplacian(rows=270, cols=480, options=opts)
        src = p.generate_code().source
        seg = src[src.index('pm_laplacian_g0_body(const'):]
        seg = seg[:seg.index('// stage')]
        loops[len(opts)] = int(re.findall(
            r'for \(int i = threadIdx.x; i < (\d+);', seg)[0])
        if len(opts) == 2:
            assert 'so_img_colour_2 = 0;' in seg
            assert p.build().so_path.endswith(".so")
        else:
            assert '& ~15;' in seg
    assert loops[1] == 32 * 64 * 32 and loops[2] == 32 * 64 * 3


def test_output_stationary_reductions():
    """Reductions whose target cell is given by plain reduction variables
    are planned output-stationary (each thread sums over the other
    reduction variables, no atomics while one tile spans them); a
    data-dependent target (the bilateral grid's intensity bin) keeps the
    scatter form."""
    from polymage_b200.apps.max_filter import build_maxfilter
    from polymage_b200.apps.bilateral_grid import build_bilateral
    plans = dict((g.plan.func.name, g.plan)
                 for g in build_maxfilter().groups
                 if g.plan.kind == 'reduction')
    assert plans['final'].gather == [0, 1, 2, None]
    assert plans['final'].tile[3] == 80          # dx spans [-26, 53]
    assert plans['vert_log'].gather == [0, 1, 2, 3]
    assert not plans['final'].privatize
    bil = [g.plan for g in build_bilateral().groups
           if g.plan.kind == 'reduction']
    assert bil and all(p.gather is None for p in bil)
    src = build_maxfilter().generate_code().source
    k = src[src.index("pm_maxfilter_g4(const"):]
    k = k[:k.index("\n}\n")]
    assert "pm_whole" in k and "acc = (acc < v) ? v : acc;" in k


def test_tile_shrinks_for_groups_over_the_shared_memory_budget():
    """The 3-D V-cycle at 8x16x64 tiles: its smoothing groups plan at the
    pipeline's tile sizes, while the restriction / interpolation groups
    that would need more shared memory than the budget are planned with
    halved tiles; option 'no_tile_shrink' refuses the plan instead."""
    from polymage_b200.apps.multigrid import build_v_cycle
    kw = dict(n=15, L=2, nu1=2, nu2=0, nuc=0, dims=3,
              tile_sizes=(8, 16, 64), group_size=1, name="Vcycle3d_t")
    p = build_v_cycle(**kw)
    tiles = [tuple(g.plan.tile) for g in p.groups
             if g.plan.kind == 'stencil']
    assert (8, 16, 64) in tiles
    assert any(t != (8, 16, 64) for t in tiles)
    for g in p.groups:
        if g.plan.kind == 'stencil':
            assert g.plan.smem_bytes <= 200 * 1024
    with pytest.raises(PlanError):
        build_v_cycle(**dict(kw, options=('no_tile_shrink',)))


def test_zero_default_reductions_start_from_a_memset():
    """A Reduction whose default is 0 (the bilateral grid) is cleared with
    cudaMemsetAsync in the single-image entry; the batched path keeps its
    init kernel."""
    from polymage_b200.apps.bilateral_grid import build_bilateral
    src = build_bilateral().generate_code().source
    launcher = src[src.index("static int launch_pm_bilateral_g0("):]
    launcher = launcher[:launcher.index("\n}\n")]
    assert "cudaMemsetAsync(L.d0.b_grid, 0, (size_t)L.d0.nbytes, s)" in \
        launcher
    assert "_init<<<" not in launcher
    assert "pm_bilateral_g0_init<<<" in src          # batches


def test_whole_channel_tiles_fold_channel_conditions():
    """With option channel_tile the camera pipe's output group computes
    the three channels of a pixel in one thread; on interior tiles the
    channel index is a literal, so the colour correction's
    Case(c == k) parts leave no runtime channel test behind and the
    channels share the demosaicked values."""
    from polymage_b200.apps import catalog
    b, kw = catalog._BUILDERS['campipe']
    assert 'channel_tile' in kw['options']
    src = b(**kw).generate_code().source
    k = src[src.index("// stage process"):]
    fast = k[k.index("if (pm_inside)"):]
    fast = fast[:fast.index("\n      }\n      else")]
    assert "== 2)" not in fast and "== 1)" not in fast
    assert fast.count("b_process[gb") == fast.count("b_process[")


def test_shared_regions_broadcast_every_declared_region():
    """Option 'shared_regions': thread 0 computes the tile's regions and
    the interior flag, every value the per-thread form declares at the
    top level is stored and read back under the same name and type."""
    from polymage_b200.codegen import _top_level_decls
    decls = _top_level_decls([
        "const int r_a_lo0 = pm_imax(a_lo0, d_a_lo0), r_a_hi0 = x;",
        "int r_b_lo0 = 0x3fffffff, r_b_hi0 = -0x3fffffff;",
        "if (!(e)) {",
        "  { const int ea = 1, eb = 2; r_b_lo0 = pm_imin(r_b_lo0, ea); }",
        "}",
        "int o_c_lo0 = (t0 == 0) ? pm_imax(a_lo0, d_c_lo0) : 5;",
        "const bool pm_inside = r_a_lo0 >= 0 && (r_b_hi0 <= 3);"])
    assert decls == [("int", "r_a_lo0"), ("int", "r_a_hi0"),
                     ("int", "r_b_lo0"), ("int", "r_b_hi0"),
                     ("int", "o_c_lo0"), ("bool", "pm_inside")]
    from polymage_b200.apps import catalog
    src = catalog.variant("harris", ("shared_regions",)).generate_code() \
        .source
    body = src[src.index("pm_harris_g0_body(const"):]
    body = body[:body.index("// stage")]
    assert "__shared__ int pm_ts1[" in body
    assert "if (threadIdx.x == 0) {" in body
    assert "const bool pm_inside = (bool)pm_ts1[" in body
    plain = catalog.variant("harris").generate_code().source
    assert "pm_ts1" not in plain


def test_storage_order_reorders_strides_only_of_intermediates():
    """Option storage_order: the named intermediate's strides follow the
    given memory order (innermost stride 1), every read of it multiplies
    its innermost index by its stride, it is not staged by TMA, and an
    invalid order is refused."""
    import re
    import pytest
    from polymage_b200.apps import catalog
    from polymage_b200.codegen import CodegenError
    p = catalog.variant("maxfilter")
    src = p.generate_code().source
    st = dict(re.findall(r'const long long (s_vert_\d) = ([^;]*);', src))
    assert st['s_vert_2'] == '1'
    assert st['s_vert_1'].startswith('s_vert_2 *')
    assert st['s_vert_0'].startswith('s_vert_1 *')
    assert st['s_vert_3'].startswith('s_vert_0 *')
    # the final maximum reads vert with a stride on its last index
    assert re.search(r'b_vert \+ \(\(long long\)\([^;]*\) \* s_vert_3\)', src)
    assert 'D.tma_vert = pm_use_tma()' not in src
    # the caller's output keeps the domain order
    assert 'const long long s_final_2 = 1;' in src
    order = [o for o in catalog.MAXFILTER['options']
             if isinstance(o, tuple) and o[0] == 'storage_order']
    bad = catalog.variant("maxfilter", [('storage_order',
                                         (('vert', (0, 1, 1, 2)),))], order)
    with pytest.raises(CodegenError):
        bad.generate_code()
