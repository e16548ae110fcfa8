"""Overlapped-tile plans for fused groups: the CUDA-target counterpart of
``fused_schedule`` / ``compute_tile_slope`` / ``overlap_tile`` /
``enable_tile_scratchpad`` (sandbox/poly_schedule.py:128-536) and of the
scratchpad decisions of storage mapping (sandbox/storage_mapping.py:461-589).

A stencil group becomes one kernel.  Each CTA owns one tile of the group's
*anchor* (its widest sink live-out) and computes, for every stage the tile
needs, exactly the region the tile depends on (its overlapped footprint):

* **Region inference.**  Walking the group's materialized stages from the
  anchor back to its inputs, a stage's region is the union over its
  consumers' regions of the range of each index expression, clamped to the
  stage's domain.  Index expressions that are monotone in one consumer
  variable (``x-2``, ``2*x+1``, ``x/2``, ``2+x/8``) map a consumer interval
  to a producer interval through its endpoints; constant indices map to a
  point; data-dependent indices (``lut(v)``, ``blury(.., zi)``) need the
  whole dimension, which must then have a compile-time extent.  The kernel
  runs the same inference at run time for its tile, so regions are exact at
  image borders for every image size.
* **Static extents.**  Shared-memory buffers need compile-time sizes.  The
  extent of every region is periodic in the tile origin (period: the
  product of the divisors in index expressions), so the planner simulates
  the inference for every residue of the origin and takes the maximum;
  repeating this at a second, far origin detects inconsistent scaling
  (e.g. a stage read at ``x`` and at ``x/2``), whose footprint grows with
  the origin and cannot be tiled -- the job ``align_and_scale``
  (sandbox/align_scale.py:93-855) does with isl.
* **Materialization.**  A stage is computed into shared memory when one of
  its consumers reads it at several points (a stencil) and recomputing it
  at each read would cost more than ``inline_budget`` expression nodes per
  consumer point; otherwise it is computed in registers at its use points
  (``Ixx = Ix*Ix`` feeding a 3x3 sum is recomputed, ``Ix`` is stored).
  Live-outs are written to HBM for the points their tile owns.
* **Input staging.**  An external producer (input image or an earlier
  group's output) read at several points per consumer point is staged into
  shared memory, by TMA when the buffer is 16-byte aligned and by
  cooperative loads otherwise; pointwise inputs are read from HBM directly.
* **Shared-memory layout.**  Buffers are placed first-fit by lifetime
  (a buffer dies after its last consumer stage), so e.g. Harris's
  ``img`` tile is dead before later stages reuse its bytes.

Alignment and scale of every stage dimension to the anchor's dimensions are
reported (``align``/``scale``) and fed to the cost model.
"""

from fractions import Fraction
import math

import numpy as np

from . import constructs as C
from .expr_ast import Value, AbstractBinaryOpNode, InbuiltFunction
from .expression import substitute_vars
from .evaluate import (is_min_max, eval_int, EvalError, monotone_dir, divisors_in,
                       try_eval_int)

SMEM_BUDGET = 200 * 1024       # bytes per CTA we allow a plan to use
DEFAULT_THREADS = 256
DEFAULT_INLINE_BUDGET = 32
MAX_PERIOD = 4096


class PlanError(Exception):
    pass


# ---------------------------------------------------------------------------
class IndexFn(object):
    """One index expression of a use, classified relative to the consumer's
    variables: ``mono`` (monotone in one consumer variable ``var`` at
    position ``cdim``), ``const`` (parameters and literals only) or ``full``
    (data dependent or otherwise unanalysable: the whole dimension)."""

    def __init__(self, expr, consumer_vars):
        self.expr = Value.numericToValue(expr)
        self.kind = 'full'
        self.var = None
        self.cdim = None
        self.dir = 0
        e = self.expr
        if is_data_dependent(e):
            return
        vs = [v for v in e.collect(C.Variable)
              if not isinstance(v, C.Parameter)]
        if not vs:
            self.kind = 'const'
            return
        if len(vs) == 1 and any(vs[0] is v for v in consumer_vars):
            d = monotone_dir(e, vs[0])
            if d in (1, -1):
                self.kind = 'mono'
                self.var = vs[0]
                self.cdim = [i for i, v in enumerate(consumer_vars)
                             if v is vs[0]][0]
                self.dir = d

    def evaluate(self, value, env):
        e = dict(env)
        if self.var is not None:
            e[self.var] = value
        return eval_int(self.expr, e)

    def key(self):
        return str(self.expr)

    def __repr__(self):
        return "<%s %s>" % (self.kind, self.expr)


def is_data_dependent(e):
    """Whether an index expression depends on data (or is not integer
    arithmetic that region inference can follow).  Max/Min of index
    arithmetic (clamped indices) are not data dependent."""
    stack = [e]
    while stack:
        n = stack.pop()
        if is_min_max(n):
            stack.extend([n.true_expression, n.false_expression])
            continue
        if isinstance(n, (C.Reference, C.Select, C.Cast, InbuiltFunction)):
            return True
        if isinstance(n, AbstractBinaryOpNode) and n.op not in ('+', '-',
                                                               '*', '/'):
            return True
        if isinstance(n, Value) and not isinstance(n.value, int):
            return True
        stack.extend(n.children())
    return False


def expr_cost(e):
    """Operations and reads of an expression (a proxy for its evaluation
    cost); index arguments of references are address arithmetic and are not
    counted, variables and literals are free."""
    n = 0
    stack = [e]
    while stack:
        x = stack.pop()
        if isinstance(x, C.Reference):
            n += 1
            continue
        if isinstance(x, (C.Variable, Value)):
            continue
        n += 1
        if hasattr(x, 'children'):
            stack.extend(x.children())
    return n


def func_cost(f):
    """Recompute cost of a stage at one point: its expressions (the Case
    conditions are cheap comparisons shared by neighbouring points and are
    not counted)."""
    from .pipe import body_parts
    total = 0
    for cond, expr, red in body_parts(f):
        total += expr_cost(expr)
    return total


# ---------------------------------------------------------------------------
class Node(object):
    """A buffer of the group plan: a live-out (``out``), a stage kept in
    shared memory (``smem``) or a staged external producer (``stage``)."""

    def __init__(self, func, role):
        self.func = func
        self.role = role              # 'out' | 'smem' | 'stage'
        self.also_smem = False        # 'out' node also read inside group
        self.uses = []                # [(consumer Node, [IndexFn])]
        self.ext = None               # static extents per dim
        self.pad_inner = None         # padded innermost extent (stage)
        self.smem_off = None
        self.smem_bytes = 0
        self.step = None              # compute step (0: staged inputs)
        self.last_step = None
        self.align = None             # anchor dim per dim (or None)
        self.scale = None             # Fraction per dim (or None)
        self.owned_map = None         # out nodes: anchor dim per own dim

    @property
    def name(self):
        return self.func.name

    @property
    def ndims(self):
        return len(self.func.domain)

    @property
    def in_smem(self):
        return self.role in ('smem', 'stage') or self.also_smem

    def __repr__(self):
        return "<node %s %s>" % (self.func.name, self.role)


class GroupPlan(object):
    """Everything the code generator needs for one fused stencil group."""
    kind = 'stencil'

    def __init__(self):
        self.funcs = []
        self.anchor = None
        self.tile = []
        self.threads = DEFAULT_THREADS
        self.nodes = []               # region-inference order (anchor 1st)
        self.node_of = {}
        self.role = {}                # func -> 'out'|'smem'|'inline'
        self.ext_role = {}            # external func -> 'stage'|'global'
        self.externals = []
        self.smem_bytes = 0
        self.period = 1
        self.steps = []               # materialized in-group funcs, order

    def describe(self):
        out = ["anchor %s tile %s threads %d smem %d B" % (
            self.anchor.name, self.tile, self.threads, self.smem_bytes)]
        for n in self.nodes:
            out.append("%-14s %-5s ext %s align %s scale %s smem@%s" % (
                n.name, n.role + ('+smem' if n.also_smem else ''), n.ext,
                n.align, [str(s) if s is not None else None
                          for s in (n.scale or [])], n.smem_off))
        inl = [f.name for f in self.funcs if self.role[f] == 'inline']
        if inl:
            out.append("inlined: " + ", ".join(inl))
        return out

    def features(self):
        """Numeric summary used by the learned cost model."""
        halo = 0
        for n in self.nodes:
            if n.ext is None or n.role == 'out':
                continue
            for d, e in enumerate(n.ext):
                if n.align and n.align[d] is not None and n.scale[d]:
                    t = self.tile[n.align[d]]
                    halo = max(halo, e - float(n.scale[d]) * t)
        pts = float(np.prod(self.tile))
        redundant = 0.0
        for n in self.nodes:
            if n.role == 'smem' and n.ext:
                redundant += float(np.prod(n.ext)) / max(pts, 1.0)
        return {
            'nstages': len(self.funcs),
            'nsmem': sum(1 for n in self.nodes if n.role == 'smem'),
            'nstage_in': sum(1 for n in self.nodes if n.role == 'stage'),
            'ninline': sum(1 for f in self.funcs
                           if self.role[f] == 'inline'),
            'tile_inner': self.tile[-1],
            'tile_outer': int(np.prod(self.tile[:-1])) if len(
                self.tile) > 1 else 1,
            'halo': halo,
            'smem_bytes': self.smem_bytes,
            'redundancy': redundant,
            'threads': self.threads,
            'cost': sum(func_cost(f) for f in self.funcs),
        }


class ReductionPlan(object):
    """Plan of a ``Reduction`` group: an init pass over the reduction's
    domain and a tiled accumulation pass over its reduction domain,
    privatized in shared memory when the tile's target footprint fits."""
    kind = 'reduction'

    def __init__(self):
        self.func = None
        self.tile = []
        self.threads = DEFAULT_THREADS
        self.target_fns = []          # per (part) list of IndexFn
        self.priv_ext = None          # static extents of privatized box
        self.privatize = False
        self.smem_bytes = 0
        self.funcs = []
        # output-stationary form: per reduction variable, the target
        # dimension it indexes (None for the variables summed over), when
        # every part targets the same cell given by plain reduction
        # variables; None otherwise
        self.gather = None

    def describe(self):
        return ["reduction %s tile %s privatize %s ext %s gather %s" % (
            self.func.name, self.tile, self.privatize, self.priv_ext,
            self.gather)]

    def features(self):
        return {'nstages': 1, 'tile_inner': self.tile[-1],
                'smem_bytes': self.smem_bytes, 'threads': self.threads}


class ConstPlan(object):
    """A ``const`` function: evaluated on the host per parameter set and
    uploaded as a table (its bit-exactness then follows the host
    compiler's, as the reference's)."""
    kind = 'const'

    def __init__(self, func):
        self.func = func
        self.funcs = [func]

    def describe(self):
        return ["const table %s" % self.func.name]

    def features(self):
        return {}


# ---------------------------------------------------------------------------
def _tile_sizes_for(pipeline, ndims, anchor=None, env=None, funcs=()):
    """Tile extent per anchor dimension: the tile sizes apply to the
    innermost dimensions, leading ones get 1.  With fewer sizes than
    dimensions, an innermost dimension of constant extent <= 4 (the
    channels of an interleaved image, [x][y][c]) is tiled whole and the
    sizes go to the dimensions before it.  A leading dimension of constant
    extent <= 4 (the channels of a planar image, [c][x][y]) can also be
    tiled whole when the group computes stages of fewer dimensions than the
    anchor (the camera pipe's red, green and blue planes feeding every
    output channel): one tile then computes them once for all channels
    instead of once per channel (option 'channel_tile'); option
    'channel_tile_all' tiles such a channel dimension whole in every group,
    so that the channels of a point share their index arithmetic and the
    lower-dimensional inputs they read."""
    ts = list(pipeline.tile_sizes)
    opt = _option(pipeline, 'tile')
    if opt is not None:
        ts = list(opt)
    if len(ts) >= ndims:
        return [int(t) for t in ts[len(ts) - ndims:]]
    tail = []
    if anchor is not None and env is not None and ndims > len(ts):
        e = _const_extent(anchor.domain[ndims - 1], env)
        if e is not None and e <= 4:
            tail = [int(e)]
    n = ndims - len(tail)
    head = [int(t) for t in ts[max(0, len(ts) - n):]]
    lead = [1] * (n - len(head))
    if lead and not tail and env is not None and \
            ('channel_tile' in pipeline.options and
             any(f.ndims < ndims for f in funcs if f is not anchor) or
             'channel_tile_all' in pipeline.options):
        e = _const_extent(anchor.domain[0], env)
        if e is not None and e <= 4:
            lead[0] = int(e)
    return lead + head + tail


def _option(pipeline, name, default=None):
    for o in pipeline.options:
        if isinstance(o, tuple) and o[0] == name:
            return o[1]
        if isinstance(o, str) and o.startswith(name + '='):
            v = o.split('=', 1)[1]
            try:
                return int(v)
            except ValueError:
                return v
    return default


def _refs_to(func, target):
    from .pipe import body_refs
    return [r for r in body_refs(func) if r.objectRef is target]


def plan_group(pipeline, group):
    """Plan of one group of the final grouping.  A stencil group whose
    tile needs more shared memory than the budget at the pipeline's tile
    sizes (the 3-D multigrid's restriction and interpolation groups at
    tiles that suit its smoothing steps) is planned with its largest tile
    dimension halved until it fits.  Grouping decisions do not see this:
    they are taken at the pipeline's tile sizes."""
    kind = group.kind
    if kind == 'const':
        return ConstPlan(group.comps[0].func)
    if kind == 'reduction':
        return plan_reduction(pipeline, group.comps)
    tile = None
    while True:
        try:
            return plan_stencil(pipeline, group.comps, tile=tile)
        except PlanError as e:
            if 'exceeds budget' not in str(e) or \
                    'no_tile_shrink' in pipeline.options:
                raise
            cur = list(tile or e.args[1])
            big = max(range(len(cur)), key=lambda d: cur[d])
            if cur[big] <= 1:
                raise
            cur[big] //= 2
            tile = cur


def check_group_plan(pipeline, comps):
    if any(c.is_const_func or c.is_reduction for c in comps):
        if len(comps) > 1:
            raise PlanError("reductions and const functions are not fused")
        return
    plan_stencil(pipeline, comps)


def plan_stencil(pipeline, comps, tile=None):
    """Plan of a fused stencil group; ``tile`` overrides the tile the
    pipeline's tile sizes give its anchor."""
    env = pipeline.int_env()
    pos = dict((c, i) for i, c in enumerate(pipeline.comps))
    comps = sorted(comps, key=lambda c: pos[c])
    funcs = [c.func for c in comps]
    ids = set(id(f) for f in funcs)
    comp_of = dict((c.func, c) for c in comps)
    mine = set(id(c) for c in comps)
    liveouts = [c.func for c in comps
                if c.is_output or any(id(k) not in mine for k in c.children)]
    consumers = dict((f, [g for g in funcs if g is not f and
                          _refs_to(g, f)]) for f in funcs)
    for f in funcs:
        if isinstance(f, C.Reduction) or f.is_const_func:
            raise PlanError("%s cannot be fused" % f.name)
        if f.getObjects(C.RandomFloat):
            raise PlanError("RandomFloat is not supported on the GPU")
    sinks = [f for f in liveouts if not consumers[f]]
    if not sinks:
        raise PlanError("group has no sink")
    order_pos = dict((f, i) for i, f in enumerate(funcs))
    anchor = max(sinks, key=lambda f: (f.ndims, order_pos[f]))
    plan = GroupPlan()
    plan.funcs = funcs
    plan.anchor = anchor
    plan.threads = int(_option(pipeline, 'threads', DEFAULT_THREADS))
    budget = int(_option(pipeline, 'inline_budget', DEFAULT_INLINE_BUDGET))
    forced_smem = set(_option(pipeline, 'materialize', []) or [])
    plan.tile = list(tile) if tile is not None else \
        _tile_sizes_for(pipeline, anchor.ndims, anchor, env, funcs)

    # ---- materialization decisions, sinks first --------------------------
    uses = {}          # func -> [(M func, [arg exprs])]
    role = {}
    for f in reversed(funcs):
        us = []
        for g in consumers[f]:
            if role[g] in ('out', 'smem'):
                for r in _refs_to(g, f):
                    us.append((g, list(r.arguments)))
            else:
                for (m, gargs) in uses[g]:
                    bind = dict(zip(g.variables, gargs))
                    for r in _refs_to(g, f):
                        us.append((m, [substitute_vars(a, bind)
                                       for a in r.arguments]))
        us = _dedupe(us)
        uses[f] = us
        if f in liveouts:
            role[f] = 'out'
            continue
        mult = _multiplicity(us)
        if mult > 1 and _disjoint_gather(us, env):
            mult = 1
        cost = func_cost(f)
        if f.name in forced_smem:
            role[f] = 'smem'
        elif mult <= 1 or cost * mult <= budget:
            role[f] = 'inline'
        else:
            role[f] = 'smem'
    plan.role = role

    # ---- external producers ---------------------------------------------
    externals = []
    ext_uses = {}
    for f in funcs:
        for r in _all_refs(f):
            x = r.objectRef
            if id(x) in ids or x is f:
                continue
            if all(x is not q for q in externals):
                externals.append(x)
    for x in externals:
        us = []
        for g in funcs:
            refs = _refs_to(g, x)
            if not refs:
                continue
            if role[g] in ('out', 'smem'):
                for r in refs:
                    us.append((g, list(r.arguments)))
            else:
                for (m, gargs) in uses[g]:
                    bind = dict(zip(g.variables, gargs))
                    for r in refs:
                        us.append((m, [substitute_vars(a, bind)
                                       for a in r.arguments]))
        ext_uses[x] = _dedupe(us)
    plan.externals = externals

    # ---- nodes -------------------------------------------------------------
    nodes = []
    node_of = {}

    def mk(f, r):
        n = Node(f, r)
        nodes.append(n)
        node_of[f] = n
        return n

    mk(anchor, 'out')
    for f in reversed(funcs):
        if f is anchor:
            continue
        if role[f] == 'out':
            n = mk(f, 'out')
            n.also_smem = bool(uses[f])
        elif role[f] == 'smem':
            mk(f, 'smem')
    stage_inputs = 'no_stage' not in pipeline.options
    # inputs read at one offset only are read straight from HBM, unless
    # option 'stage_pointwise' asks for them to be staged by TMA too (the
    # copy is then in flight while the tile's other stages compute)
    min_mult = 1 if 'stage_pointwise' in pipeline.options else 2
    for x in externals:
        us = ext_uses[x]
        want = stage_inputs and _multiplicity(us) >= min_mult and \
            not x.is_const_func
        if want:
            for m, args in us:
                for a, dom in zip(args, x.domain):
                    fn = IndexFn(a, m.variables)
                    if fn.kind == 'full' and _const_extent(dom, env) is None:
                        want = False
        plan.ext_role[x] = 'stage' if want else 'global'
        if want:
            mk(x, 'stage')
    # externals read straight from HBM get a footprint node too (never
    # materialized): the kernel uses it to prove that an interior tile's
    # reads stay inside the buffer before taking its unguarded fast path
    for x in externals:
        if plan.ext_role[x] == 'global':
            mk(x, 'global')
    # stages computed in registers get a footprint node as well: the kernel
    # checks their Case conditions against it to drop them on tiles where
    # they hold everywhere
    for f in reversed(funcs):
        if role[f] == 'inline' and uses[f]:
            mk(f, 'inline')

    # attach uses as (node, IndexFn list)
    for n in nodes:
        src = ext_uses[n.func] if n.role in ('stage', 'global') \
            else uses[n.func]
        for m, args in src:
            if m not in node_of:
                raise PlanError("internal: consumer %s not materialized"
                                % m.name)
            fns = [IndexFn(a, m.variables) for a in args]
            n.uses.append((node_of[m], fns))
        for fnl in n.uses:
            for fn, dom in zip(fnl[1], n.func.domain):
                if fn.kind == 'full' and n.in_smem and \
                        _const_extent(dom, env) is None:
                    raise PlanError("%s: data-dependent access to a "
                                    "dimension of parametric extent"
                                    % n.name)
    # out nodes other than the anchor: positional alignment
    for n in nodes:
        if n.role != 'out':
            continue
        if n.ndims > anchor.ndims:
            raise PlanError("live-out %s has more dimensions than the "
                            "anchor %s" % (n.name, anchor.name))
        off = anchor.ndims - n.ndims
        n.owned_map = [off + d for d in range(n.ndims)]
    for n in nodes:
        # materialized consumers read only where their Case holds
        n.case_box = case_box(n.func) if n.role in ('out', 'smem') else None
    plan.nodes = nodes
    plan.node_of = node_of

    # ---- steps (order in which materialized stages are computed) ---------
    steps = [f for f in funcs if role[f] in ('out', 'smem')]
    plan.steps = steps
    for n in nodes:
        n.step = 0 if n.role in ('stage', 'global', 'inline') else \
            steps.index(n.func) + 1
    for n in nodes:
        last = n.step
        for m, _ in n.uses:
            last = max(last, m.step)
        n.last_step = last

    _static_extents(plan, env)
    _alignment(plan, env)
    _layout_smem(plan, tight=('tight_stage' in pipeline.options), env=env,
                 prefetch=('prefetch' in pipeline.options))
    if plan.smem_bytes > int(_option(pipeline, 'smem_budget', SMEM_BUDGET)):
        raise PlanError("shared memory %d B exceeds budget" %
                        plan.smem_bytes, list(plan.tile))
    return plan


def _all_refs(f):
    from .pipe import body_refs
    return body_refs(f)


def _dedupe(us):
    seen = set()
    out = []
    for m, args in us:
        k = (id(m), tuple(str(a) for a in args))
        if k in seen:
            continue
        seen.add(k)
        out.append((m, args))
    return out


def _multiplicity(us):
    cnt = {}
    for m, args in us:
        cnt[id(m)] = cnt.get(id(m), 0) + 1
    return max(cnt.values()) if cnt else 0


def _disjoint_gather(us, env):
    """Whether a producer read at several points per consumer point is
    still read at most once per point overall: each consumer reads it at
    tuples that agree, position for position, on distinct plain consumer
    variables and differ only in integer constants elsewhere (the
    bilateral grid's ``filtered`` reading ``interpolated(0, x, y)`` and
    ``interpolated(1, x, y)``), and every consumer variable left out of
    those positions ranges over one value.  Recomputing such a producer at
    its reads then costs what storing it would, without the shared-memory
    round trip."""
    by = {}
    for m, args in us:
        by.setdefault(id(m), (m, []))[1].append(args)
    for m, tuples in by.values():
        if len(tuples) < 2:
            continue
        used = []
        for pos in range(len(tuples[0])):
            col = [Value.numericToValue(t[pos]) for t in tuples]
            if all(str(c) == str(col[0]) for c in col):
                v = col[0]
                if not isinstance(v, C.Variable) or \
                        isinstance(v, C.Parameter) or \
                        any(v is u for u in used):
                    return False
                used.append(v)
            elif not all(isinstance(c, Value) and isinstance(c.value, int)
                         for c in col):
                return False
        if len(set(tuple(str(a) for a in t) for t in tuples)) != \
                len(tuples):
            return False
        for v, dom in zip(m.variables, m.domain):
            if any(v is u for u in used):
                continue
            if _const_extent(dom, env) != 1:
                return False
    return True


def _const_extent(dom, env):
    """Extent of an interval if it does not depend on parameters."""
    env2 = dict((k, v * 3 + 17) for k, v in env.items())
    a = try_eval_int(dom.upperBound - dom.lowerBound + 1, env)
    b = try_eval_int(dom.upperBound - dom.lowerBound + 1, env2)
    if a is None or a != b:
        return None
    return a


def _domain_vals(func, env):
    out = []
    for d in func.domain:
        out.append((eval_int(d.lowerBound, env), eval_int(d.upperBound, env)))
    return out


def case_box(func):
    """Per-dimension (lower-bound exprs, upper-bound exprs) of the single
    box-shaped Case of ``func`` (None when it has several pieces, a plain
    expression, or a condition that is not a box).  A consumer only reads
    its producers where its Case holds, so footprints are computed over
    the consumer's region intersected with this box."""
    from .pipe import body_parts
    from .bounds import part_boxes
    parts = body_parts(func)
    if len(parts) != 1 or parts[0][0] is None or parts[0][2] is not None:
        return None
    boxes = part_boxes(func)
    if len(boxes) != 1 or not boxes[0][0].exact:
        return None
    b = boxes[0][0]
    return [(b.lo[v], b.hi[v]) for v in func.variables]


def case_restricted(node, region, env, constant_only=False):
    """A node's region intersected with its Case box.  With
    ``constant_only`` (static-extent simulation at far tile origins) only
    bounds that do not depend on parameters are applied."""
    lo, hi = region
    cb = getattr(node, 'case_box', None)
    if not cb:
        return lo, hi
    lo = list(lo)
    hi = list(hi)
    env2 = dict((k, v * 3 + 17) for k, v in env.items())
    for d, (los, his) in enumerate(cb):
        for e in los:
            v = try_eval_int(e, env)
            if v is None or (constant_only and try_eval_int(e, env2) != v):
                continue
            lo[d] = np.maximum(lo[d], v)
        for e in his:
            v = try_eval_int(e, env)
            if v is None or (constant_only and try_eval_int(e, env2) != v):
                continue
            hi[d] = np.minimum(hi[d], v)
    return lo, hi


def infer_regions(plan, anchor_box, env, clamp=True, tile_first=None):
    """Region of every node for one tile (numpy-vectorizable: box bounds may
    be arrays).  ``anchor_box``: [(lo, hi)] per anchor dim.  ``tile_first``:
    per anchor dim, whether the tile is the first along that dim (used for
    ownership of lower-dimensional live-outs)."""
    if not clamp:
        # unclamped regions model interior tiles far from every border:
        # parameters are taken huge so that indices clamped to a
        # parameter-dependent bound (min/max) behave as in the interior
        env = dict((k, 1 << 40) for k in env)
    regions = {}
    big = 1 << 60
    for n in plan.nodes:
        dom = _domain_vals(n.func, env)
        nd = n.ndims
        if n.func is plan.anchor:
            lo = [anchor_box[d][0] for d in range(nd)]
            hi = [anchor_box[d][1] for d in range(nd)]
        elif n.role == 'out':
            lo = []
            hi = []
            for d in range(nd):
                k = n.owned_map[d]
                lo.append(anchor_box[k][0])
                hi.append(anchor_box[k][1])
            # unmatched leading anchor dims: only the first tile owns
            if tile_first is not None:
                for k in range(plan.anchor.ndims - nd):
                    if not tile_first[k]:
                        lo = [big] * nd
                        hi = [-big] * nd
            if not clamp:
                lo = [np.asarray(l) for l in lo]
        else:
            lo = [big] * nd
            hi = [-big] * nd
        if n.role == 'out' and n.func is not plan.anchor and clamp:
            lo = [np.maximum(l, dom[d][0]) for d, l in enumerate(lo)]
            hi = [np.minimum(h, dom[d][1]) for d, h in enumerate(hi)]
        for m, fns in n.uses:
            mlo, mhi = case_restricted(m, regions[m.func], env,
                                       constant_only=not clamp)
            nonempty = np.ones_like(np.asarray(mlo[0]), dtype=bool) \
                if mlo else True
            for d in range(len(mlo)):
                nonempty = nonempty & (np.asarray(mlo[d]) <=
                                       np.asarray(mhi[d]))
            for d, fn in enumerate(fns):
                if fn.kind == 'mono':
                    a = fn.evaluate(mlo[fn.cdim], env)
                    b = fn.evaluate(mhi[fn.cdim], env)
                    a, b = np.minimum(a, b), np.maximum(a, b)
                elif fn.kind == 'const':
                    a = b = fn.evaluate(0, env)
                else:
                    a, b = dom[d]
                lo[d] = np.where(nonempty, np.minimum(lo[d], a), lo[d])
                hi[d] = np.where(nonempty, np.maximum(hi[d], b), hi[d])
        if clamp:
            lo = [np.maximum(l, dom[d][0]) for d, l in enumerate(lo)]
            hi = [np.minimum(h, dom[d][1]) for d, h in enumerate(hi)]
        regions[n.func] = (lo, hi)
    return regions


def _grid_lo(plan):
    """Per anchor dim, the first tile origin when it is a constant (the
    smallest lower bound of the live-outs' domains along that dim, as the
    generated descriptor filler computes it), else None."""
    from .codegen import _const_int
    na = plan.anchor.ndims
    out = [None] * na
    seen = [False] * na
    ok = [True] * na
    for n in plan.nodes:
        if n.role != 'out' and n.func is not plan.anchor:
            continue
        for d, dom in enumerate(n.func.domain):
            k = d if n.func is plan.anchor else n.owned_map[d]
            v = _const_int(dom.lowerBound)
            if v is None:
                ok[k] = False
                continue
            out[k] = v if not seen[k] else min(out[k], v)
            seen[k] = True
    return [out[k] if ok[k] and seen[k] else None for k in range(na)]


def _static_extents(plan, env):
    # period of every node's region in the tile origin: the lcm, over the
    # chains of uses from the anchor, of the product of the divisors met
    per = {}
    capped = False
    divs = []
    for n in plan.nodes:
        p = 1
        for m, fns in n.uses:
            q = per.get(m.func, 1)
            for fn in fns:
                if fn.kind == 'mono':
                    for dv in divisors_in(fn.expr):
                        q *= dv
                        divs.append(dv)
            p = p * q // math.gcd(p, q)
        if p > MAX_PERIOD:
            capped = True
            p = MAX_PERIOD
        per[n.func] = p
    period = 1
    for p in per.values():
        period = period * p // math.gcd(period, p)
        if period > MAX_PERIOD:
            capped = True
            period = MAX_PERIOD
    plan.period = period
    exts = []
    adom = _domain_vals(plan.anchor, env)
    glo = _grid_lo(plan)
    for base in (period * (1 << 22), period * (1 << 23) + period * 7):
        # anchor dims of constant extent: their actual tiles; parametric
        # dims: the residues of the origin (mod the period) that tiles can
        # have, far from any border -- all of them unless the tile grid
        # starts at a constant, when only glo + j*tile occur
        axes = []
        for k, t in enumerate(plan.tile):
            if _const_extent(plan.anchor.domain[k], env) is not None:
                lo0, hi0 = adom[k]
                axes.append(np.arange(lo0, hi0 + 1, t, dtype=np.int64))
            elif glo[k] is not None:
                res = sorted(set((glo[k] + j * t) % period
                                 for j in range(period)))
                axes.append(base + np.asarray(res, dtype=np.int64))
            else:
                axes.append(base + np.arange(period, dtype=np.int64))
        grids = np.meshgrid(*axes, indexing='ij')
        box = []
        for k, t in enumerate(plan.tile):
            lo = grids[k].ravel()
            hi = lo + t - 1
            if _const_extent(plan.anchor.domain[k], env) is not None:
                hi = np.minimum(hi, adom[k][1])
            box.append((lo, hi))
        regs = infer_regions(plan, box, env, clamp=False)
        cur = {}
        for n in plan.nodes:
            lo, hi = regs[n.func]
            e = []
            dom = _domain_vals(n.func, env)
            for d in range(n.ndims):
                ext = np.max(np.asarray(hi[d]) - np.asarray(lo[d]) + 1)
                # 'full' dims: clamp to the (constant) domain extent
                dext = dom[d][1] - dom[d][0] + 1
                full = any(fns[d].kind == 'full' for _, fns in n.uses)
                if full:
                    ext = max(min(int(ext), dext), 1)
                e.append(int(max(ext, 1)))
            cur[n.func] = e
        exts.append(cur)
    for n in plan.nodes:
        a, b = exts[0][n.func], exts[1][n.func]
        if a != b:
            if n.role == 'stage':
                # an input read at inconsistent scales is not staged
                n.role = 'global'
                plan.ext_role[n.func] = 'global'
            elif n.role not in ('global', 'inline'):
                raise PlanError("inconsistent scaling: footprint of %s "
                                "grows with the tile origin" % n.name)
        if n.func is plan.anchor or n.role == 'out' and not n.also_smem:
            n.ext = [min(x, t) for x, t in
                     zip(a, plan.tile[plan.anchor.ndims - n.ndims:])]
        else:
            n.ext = a
        if capped:
            n.ext = [x + 2 for x in n.ext]


def _alignment(plan, env):
    """Anchor dimension and scale of every node dimension, from the
    composed monotone index functions (slope measured over a long span)."""
    K = 1 << 16
    base = 1 << 20
    # interior behaviour: parameter-dependent clamps must not bind
    env = dict((k, 1 << 40) for k in env)
    for n in plan.nodes:
        n.align = [None] * n.ndims
        n.scale = [None] * n.ndims
        if n.func is plan.anchor:
            n.align = list(range(n.ndims))
            n.scale = [Fraction(1)] * n.ndims
            continue
    # propagate in node order (consumers come first)
    for n in plan.nodes:
        if n.func is plan.anchor:
            continue
        if n.role == 'out':
            n.align = list(n.owned_map)
            n.scale = [Fraction(1)] * n.ndims
        for m, fns in n.uses:
            for d, fn in enumerate(fns):
                if fn.kind != 'mono' or m.align[fn.cdim] is None:
                    continue
                try:
                    a = fn.evaluate(base, env)
                    b = fn.evaluate(base + K, env)
                except EvalError:
                    continue
                s = Fraction(b - a, K).limit_denominator(256) * \
                    m.scale[fn.cdim]
                if n.align[d] is None:
                    n.align[d] = m.align[fn.cdim]
                    n.scale[d] = s
                elif n.align[d] == m.align[fn.cdim] and n.scale[d] != s:
                    if n.role in ('global', 'inline'):
                        n.scale[d] = None      # read at several scales
                        continue
                    raise PlanError("inconsistent scaling of %s" % n.name)


def _layout_smem(plan, tight=False, env=None, prefetch=False):
    """Shared-memory buffers, placed first-fit by lifetime.  A staged
    input's rows carry the slack a TMA box needs when its origin is
    rounded down to 16 bytes; with ``tight`` (option 'tight_stage') an
    input whose innermost dimension is staged whole and is narrower than
    16 bytes (the channels of an interleaved uint8 image), which no tensor
    map can describe, gets rows of exactly that width: its origin offset
    is then always 0 and the cooperative loads cover only used bytes.

    With ``prefetch`` (option 'prefetch': a CTA loads its next tile's
    staged inputs while it computes the current tile) staged inputs live
    for the whole tile, so that no stage buffer shares their bytes, and
    get a second copy ``plan.stage_delta`` bytes above the first; the
    tiles of a CTA alternate between the two copies."""
    bufs = []
    for n in plan.nodes:
        if not n.in_smem:
            n.smem_bytes = 0
            continue
        es = n.func.typ.size()
        ext = list(n.ext)
        n.tight = False
        if n.role == 'stage':
            al = max(1, 16 // es)
            whole = env is not None and _const_extent(
                n.func.domain[-1], env) == ext[-1]
            if tight and whole and ext[-1] < al:
                w = ext[-1]
                n.tight = True
            else:
                w = ((ext[-1] + al - 1 + al - 1) // al) * al
            n.pad_inner = w
            ext[-1] = w
        elif es == 4 and ext[-1] % 4 and ext[-1] > 4:
            # rows of whole 16-byte chunks, so that the interior path can
            # read four consecutive points with one vector load
            n.pad_inner = ((ext[-1] + 3) // 4) * 4
            ext[-1] = n.pad_inner
        nbytes = es
        for e in ext:
            nbytes *= e
        n.smem_bytes = ((nbytes + 127) // 128) * 128
        bufs.append(n)
    plan.stage_delta = 0
    staged = [n for n in bufs if n.role == 'stage'] if prefetch else []
    end = max([n.last_step for n in bufs] or [0])

    def life(q):
        return (q.step, end if q in staged else q.last_step)

    placed = []
    total = 0
    for n in sorted(bufs, key=lambda q: (q.step, -q.smem_bytes)):
        off = 0
        while True:
            clash = None
            for p in placed:
                overlap_t = not (life(p)[1] < life(n)[0] or
                                 life(n)[1] < life(p)[0])
                overlap_m = off < p.smem_off + p.smem_bytes and \
                    p.smem_off < off + n.smem_bytes
                if overlap_t and overlap_m:
                    clash = p
                    break
            if clash is None:
                break
            off = clash.smem_off + clash.smem_bytes
        n.smem_off = off
        placed.append(n)
        total = max(total, off + n.smem_bytes)
    if staged:
        plan.stage_delta = ((total + 127) // 128) * 128
        total = plan.stage_delta + max(n.smem_off + n.smem_bytes
                                       for n in staged)
    plan.smem_bytes = total + 128       # + mbarrier / flags area


# ---------------------------------------------------------------------------
def _gather_map(pipeline, f, rvars):
    """Target dimension of each reduction variable when the reduction is
    output-stationary: every part accumulates with the same operator into
    the cell whose coordinates are plain reduction variables, the same
    ones in every part and each at most once.  The other reduction
    variables are then summed over inside one thread, with no atomics
    (option 'no_gather' keeps the scatter form).  None otherwise."""
    from .pipe import body_parts
    if 'no_gather' in pipeline.options:
        return None
    parts = body_parts(f)
    if len(set(red.op_type for _, _, red in parts)) != 1:
        return None
    tmap = None
    for _, _, red in parts:
        m = [None] * len(rvars)
        for t, a in enumerate(red.accumulate_ref.arguments):
            hit = [i for i, v in enumerate(rvars) if a is v]
            if len(hit) != 1 or m[hit[0]] is not None:
                return None
            m[hit[0]] = t
        if tmap is not None and m != tmap:
            return None
        tmap = m
    return tmap


def plan_reduction(pipeline, comps):
    from .pipe import body_parts
    if len(comps) != 1:
        raise PlanError("reductions are not fused")
    f = comps[0].func
    env = pipeline.int_env()
    plan = ReductionPlan()
    plan.func = f
    plan.funcs = [f]
    plan.threads = int(_option(pipeline, 'threads', DEFAULT_THREADS))
    rvars = f.reductionVariables
    plan.tile = _tile_sizes_for(pipeline, len(rvars))
    # option ('red_tile:<name>', tile) for one reduction, else
    # ('red_tile', tile) for all of them
    ts = _option(pipeline, 'red_tile:' + f.name)
    if ts is None:
        ts = _option(pipeline, 'red_tile')
    if ts is not None:
        plan.tile = list(ts)[-len(rvars):]
    fns_all = []
    for cond, expr, red in body_parts(f):
        if red is None:
            raise PlanError("reduction %s has a non-Reduce piece" % f.name)
        fns_all.append([IndexFn(a, rvars)
                        for a in red.accumulate_ref.arguments])
    plan.target_fns = fns_all
    plan.gather = _gather_map(pipeline, f, rvars)
    if plan.gather is not None:
        # each thread owns target cells and loops over the other reduction
        # variables: their tile is their whole range at the parameter
        # estimates (a call with a longer range splits it over tiles,
        # which then combine with atomics)
        for d, t in enumerate(plan.gather):
            if t is None:
                dom = f.reductionDomain[d]
                ext = try_eval_int(dom.upperBound - dom.lowerBound + 1, env)
                if ext is not None:
                    plan.tile[d] = max(plan.tile[d], min(int(ext), 1 << 20))
        return plan
    # privatized footprint of one tile, by simulation over a period
    divs = []
    for fns in fns_all:
        for fn in fns:
            if fn.kind == 'mono':
                divs += divisors_in(fn.expr)
    period = 1
    for q in divs:
        period = period * q // math.gcd(period, q)
    period = min(period, MAX_PERIOD)
    dom = _domain_vals(f, env)
    ok = True
    ext = [1] * f.ndims
    r = np.arange(period, dtype=np.int64)
    base = period * (1 << 22)
    for d in range(f.ndims):
        lo = np.full(period, 1 << 60)
        hi = np.full(period, -(1 << 60))
        for fns in fns_all:
            fn = fns[d]
            if fn.kind == 'mono':
                t = plan.tile[fn.cdim]
                a = fn.evaluate(base + r, env)
                b = fn.evaluate(base + r + t - 1, env)
                lo = np.minimum(lo, np.minimum(a, b))
                hi = np.maximum(hi, np.maximum(a, b))
            elif fn.kind == 'const':
                v = fn.evaluate(0, env)
                lo = np.minimum(lo, v)
                hi = np.maximum(hi, v)
            else:
                ce = _const_extent(f.domain[d], env)
                if ce is None:
                    ok = False
                    break
                lo = np.minimum(lo, dom[d][0])
                hi = np.maximum(hi, dom[d][1])
        if not ok:
            break
        ext[d] = int(np.max(hi - lo + 1))
    plan.priv_ext = ext
    nbytes = f.typ.size() * int(np.prod(ext))
    plan.privatize = ok and nbytes <= 64 * 1024 and \
        'no_privatize' not in pipeline.options and \
        f.typ.size() in (4, 8)
    plan.smem_bytes = nbytes if plan.privatize else 0
    return plan
