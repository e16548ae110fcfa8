"""Pipeline IR and pass driver.

``Pipeline`` mirrors the reference's pass sequence (sandbox/pipe.py:595-759):
collect the functions reachable from the outputs (``get_funcs`` :101), clone
them, build one compute object per function (``ComputeObject`` :123) and one
initial group per compute object (``Group`` :354), run the bounds check
(bounds.py), the inline pass (inline.py), automatic grouping (grouping.py),
order the groups level by level (schedule.py), then compute liveness
(liveness.py) and map storage (storage_mapping.py).

Where the reference builds isl schedules and an isl AST per group, this
backend builds a ``GroupPlan`` (tiling.py): overlapped-tile geometry, region
inference and shared-memory layout for one CUDA kernel per fused group.
``generate_code`` returns the CUDA translation unit (codegen.py) and
``build`` compiles it into a shared library whose ``pipeline_<name>`` entry
point has the reference's C ABI.
"""

import logging

from .expr_ast import Value
from . import constructs as C
from .expression import rebuild, rebuild_cond
from .evaluate import eval_int

LOG = logging.getLogger("polymage_b200.pipe")


class PipelineError(Exception):
    pass


# ---------------------------------------------------------------------------
def body_parts(func):
    """(condition or None, expression, reduce or None) for every piece of a
    function's definition."""
    out = []
    for p in func.defn:
        if isinstance(p, C.Case):
            e = p.expression
            if isinstance(e, C.Reduce):
                out.append((p.condition, e.expression, e))
            else:
                out.append((p.condition, e, None))
        elif isinstance(p, C.Reduce):
            out.append((None, p.expression, p))
        else:
            out.append((None, p, None))
    return out


def body_refs(func):
    """All references appearing in a function's definition, conditions
    included.  The accumulation target of a ``Reduce`` is not a read and is
    excluded, but references inside its index arguments are included."""
    refs = []
    for cond, expr, red in body_parts(func):
        if cond is not None:
            refs += cond.collect(C.Reference)
        refs += expr.collect(C.Reference)
        if red is not None:
            for a in red.accumulate_ref.arguments:
                refs += a.collect(C.Reference)
    if isinstance(func, C.Reduction):
        refs += func.default.collect(C.Reference)
    return refs


def get_funcs(outputs):
    """Functions and images reachable from ``outputs``.

    Returns ``(funcs, images, parents)`` with ``funcs`` in a deterministic
    topological order (producers first) and ``parents[f]`` the distinct
    functions/images ``f`` reads (sandbox/pipe.py:101-121)."""
    parents = {}
    order = []
    images = []
    visiting = set()
    done = set()

    def visit(f):
        if id(f) in done:
            return
        if isinstance(f, C.Image):
            done.add(id(f))
            images.append(f)
            return
        if id(f) in visiting:
            raise PipelineError("cyclic dependence through " + f.name)
        if not isinstance(f, C.Function):
            raise PipelineError("%r is not a Function" % (f,))
        visiting.add(id(f))
        ps = []
        for r in body_refs(f):
            o = r.objectRef
            if o is f:
                continue
            if all(o is not q for q in ps):
                ps.append(o)
        parents[f] = ps
        for p in sorted(ps, key=lambda q: q.name):
            visit(p)
        visiting.discard(id(f))
        done.add(id(f))
        order.append(f)

    for o in sorted(outputs, key=lambda q: q.name):
        visit(o)
    return order, images, parents


def collect_params(funcs, images):
    params = []

    def add(ps):
        for p in ps:
            if all(p is not q for q in params):
                params.append(p)
    for f in funcs:
        add(f.getObjects(C.Parameter))
        if isinstance(f, C.Reduction):
            for d in f.reductionDomain:
                add(d.collect(C.Parameter))
    for im in images:
        for d in im.dimensions:
            add(d.collect(C.Parameter))
    return params


def clone_functions(funcs):
    """Clone functions so that passes may rewrite bodies without touching
    the user's objects.  Images are shared, not cloned."""
    cmap = {}
    for f in funcs:
        if isinstance(f, C.Reduction):
            g = C.Reduction((list(f.variables), list(f.domain)),
                            (list(f.reductionVariables),
                             list(f.reductionDomain)), f.typ, f.name)
        else:
            g = C.Function((list(f.variables), list(f.domain)), f.typ,
                           f.name, "const" if f.is_const_func else "")
        cmap[f] = g

    def leaf(n):
        if isinstance(n, C.Reference) and n.objectRef in cmap:
            return C.Reference(cmap[n.objectRef],
                               [rebuild(a, leaf) for a in n.arguments])
        return None

    def rb(e):
        return rebuild(e, leaf)

    for f in funcs:
        g = cmap[f]
        parts = []
        for p in f.defn:
            if isinstance(p, C.Case):
                e = p.expression
                if isinstance(e, C.Reduce):
                    e = C.Reduce(rb(e.accumulate_ref), rb(e.expression),
                                 e.op_type)
                else:
                    e = rb(e)
                parts.append(C.Case(rebuild_cond(p.condition, leaf), e))
            elif isinstance(p, C.Reduce):
                parts.append(C.Reduce(rb(p.accumulate_ref), rb(p.expression),
                                      p.op_type))
            else:
                parts.append(rb(p))
        g.defn = parts
        if isinstance(f, C.Reduction):
            g.default = rb(f.default)
    return cmap


# ---------------------------------------------------------------------------
class ComputeObject(object):
    """One function of the pipeline with its DAG neighbours
    (sandbox/pipe.py:123-352)."""

    def __init__(self, func, is_output):
        self.func = func
        self.is_output = is_output
        self.parents = []      # ComputeObjects read by this one
        self.children = []     # ComputeObjects reading this one
        self.images = []       # Images read by this one
        self.group = None
        self.level = 0

    @property
    def name(self):
        return self.func.name

    @property
    def is_const_func(self):
        return self.func.is_const_func

    @property
    def is_reduction(self):
        return isinstance(self.func, C.Reduction)

    def __repr__(self):
        return "<comp %s>" % self.func.name


class Group(object):
    """A set of compute objects fused into one kernel
    (sandbox/pipe.py:354-594)."""
    _count = 0

    def __init__(self, comps):
        self.comps = list(comps)
        for c in self.comps:
            c.group = self
        self.parents = []
        self.children = []
        self.plan = None
        self.level = 0
        Group._count += 1
        self.uid = Group._count

    @property
    def name(self):
        return "_".join(c.func.name for c in self.comps)

    @property
    def kind(self):
        if any(c.is_const_func for c in self.comps):
            return 'const'
        if any(c.is_reduction for c in self.comps):
            return 'reduction'
        return 'stencil'

    @property
    def image_refs(self):
        out = []
        for c in self.comps:
            for im in c.images:
                if all(im is not q for q in out):
                    out.append(im)
        return out

    def find_parents_children(self):
        mine = set(id(c) for c in self.comps)
        ps, cs = [], []
        for c in self.comps:
            for p in c.parents:
                if id(p) not in mine and p.group not in ps:
                    ps.append(p.group)
            for ch in c.children:
                if id(ch) not in mine and ch.group not in cs:
                    cs.append(ch.group)
        self.parents, self.children = ps, cs

    def liveouts(self):
        """Compute objects whose values leave the group."""
        mine = set(id(c) for c in self.comps)
        return [c for c in self.comps
                if c.is_output or any(id(ch) not in mine
                                      for ch in c.children)]

    def __repr__(self):
        return "<group %s>" % self.name


# ---------------------------------------------------------------------------
class Pipeline(object):
    """A compiled pipeline.  Constructed by ``compiler.buildPipeline``."""

    def __init__(self, _outputs, _param_estimates=(), _param_constraints=(),
                 _grouping=(), _group_size=5, _inline_directives=(),
                 _tile_sizes=(16, 16, 16), _size_threshold=200 * 200,
                 _name=None, _options=(), _ctx=None):
        from . import bounds, inline, grouping, schedule, liveness
        from . import storage_mapping, tiling

        self._name = _name if _name is not None else "pipe"
        self._options = list(_options)
        self._group_size = _group_size
        self._tile_sizes = list(_tile_sizes)
        self._size_threshold = _size_threshold
        self._param_constraints = list(_param_constraints)
        self._inline_directives = list(_inline_directives)
        self._grouping = list(_grouping)

        for o in _outputs:
            if isinstance(o, C.Image) or not isinstance(o, C.Function):
                raise PipelineError("pipeline outputs must be Functions")

        orig_funcs, images, _ = get_funcs(list(_outputs))
        self._clone_map = clone_functions(orig_funcs)
        self._orig_outputs = list(_outputs)
        self._outputs = [self._clone_map[o] for o in _outputs]
        funcs, images, parents = get_funcs(self._outputs)
        self._inputs = images
        self._params = collect_params(funcs, images)
        self._param_estimates = self._make_estimates(_param_estimates,
                                                     _param_constraints)

        # compute objects
        self._func_map = {}
        self._comps = []
        for f in funcs:
            comp = ComputeObject(f, any(f is o for o in self._outputs))
            self._func_map[f] = comp
            self._comps.append(comp)
        for f in funcs:
            comp = self._func_map[f]
            for p in parents[f]:
                if isinstance(p, C.Image):
                    comp.images.append(p)
                else:
                    pc = self._func_map[p]
                    comp.parents.append(pc)
                    pc.children.append(comp)

        # the passes, in the reference's order
        bounds.bounds_check_pass(self)
        inline.inline_pass(self)
        if 'separable' in self._options:
            from .separable import separable_pass
            self._separable = separable_pass(self)
        self._groups = [Group([c]) for c in self._comps]
        self._refresh_groups()
        if self._grouping:
            grouping.manual_group(self, self._grouping)
        else:
            grouping.auto_group(self)
            ms = tiling._option(self, 'merge_small')
            if ms:
                grouping.merge_small(self, int(ms))
            if 'fuse_all' in self._options:
                grouping.fuse_all(self)
        schedule.schedule_groups(self)
        for g in self._groups:
            g.plan = tiling.plan_group(self, g)
        liveness.liveness_for_pipe_outputs(self)
        storage_mapping.map_storage(self)

    # ---- helpers -----------------------------------------------------------
    def _make_estimates(self, estimates, constraints):
        env = {}
        for p, v in estimates:
            env[p] = v
        for c in constraints:
            if c.conditional == '==' and isinstance(c.lhs, C.Parameter):
                r = c.rhs
                if isinstance(r, Value):
                    env.setdefault(c.lhs, r.value)
        for p in self._params:
            if p not in env:
                env[p] = 1024 if p.typ in (C.Int, C.UInt, C.Long,
                                          C.Short) else 1.0
        return env

    def _refresh_groups(self):
        for g in self._groups:
            g.find_parents_children()

    def merge_groups(self, g1, g2):
        """Fuse two groups into a new one (sandbox/pipe.py:1019-1030)."""
        comps = [c for c in self._comps
                 if c.group is g1 or c.group is g2]
        ng = Group(comps)
        self._groups = [g for g in self._groups if g is not g1 and
                        g is not g2]
        self._groups.append(ng)
        self._refresh_groups()
        return ng

    def drop_comp(self, comp):
        for p in comp.parents:
            p.children = [c for c in p.children if c is not comp]
        for ch in comp.children:
            ch.parents = [c for c in ch.parents if c is not comp]
        self._comps = [c for c in self._comps if c is not comp]
        self._func_map.pop(comp.func, None)

    def estimate(self, expr):
        return eval_int(expr, self.int_env())

    def int_env(self):
        return dict((p, int(v)) for p, v in self._param_estimates.items()
                    if p.typ not in (C.Float, C.Double))

    # ---- public properties (reference names) -----------------------------
    @property
    def name(self):
        return self._name

    @property
    def func_map(self):
        return self._func_map

    @property
    def comps(self):
        return self._comps

    @property
    def groups(self):
        return self._groups

    @property
    def outputs(self):
        return list(self._outputs)

    @property
    def inputs(self):
        return list(self._inputs)

    @property
    def options(self):
        return list(self._options)

    @property
    def group_size(self):
        return self._group_size

    @property
    def tile_sizes(self):
        return list(self._tile_sizes)

    def get_parameters(self):
        return list(self._params)

    def ordered_params(self):
        """Parameters, inputs and outputs in the C-ABI order: each list
        sorted by name with Python string order
        (sandbox/apps/../utils.py:87-100, codegen.py:957-999)."""
        params = sorted(self._params, key=lambda p: p.name)
        inputs = sorted(self._inputs, key=lambda f: f.name)
        outputs = sorted(self._outputs, key=lambda f: f.name)
        return params, inputs, outputs

    def describe(self):
        lines = ["pipeline %s" % self._name]
        for g in self._groups:
            lines.append("  group %s [%s]" % (g.name, g.kind))
            if g.plan is not None:
                lines.extend("    " + l for l in g.plan.describe())
        return "\n".join(lines)

    @property
    def pipeline_graph(self):
        """The grouped stage graph (``draw_pipeline_graph``), as the
        reference's tests read it (sandbox/tests/test_grouping.py:47)."""
        return self.draw_pipeline_graph()

    def draw_pipeline_graph(self):
        """The stage graph with its fused groups (the reference's
        ``Pipeline.draw_pipeline_graph``, sandbox/pipe.py:901-932): one box
        per stage, bold for live-outs and filled otherwise, coloured by
        HBM storage slot; one dashed cluster per group labelled with its
        launch order; an edge from each producer to each consumer.
        Returned as a ``PipelineGraph`` whose ``string()`` is Graphviz DOT
        text and ``write(path)`` writes it (the reference returns a
        pygraphviz graph with the same two methods)."""
        slot = getattr(self, '_storage_assign', {})
        palette = ("lightblue", "lightpink", "palegreen", "khaki",
                   "lightsalmon", "plum", "lightcyan", "wheat",
                   "lightgrey", "aquamarine", "thistle", "peachpuff")
        q = lambda n: '"%s"' % n.replace('"', r'\"')
        lines = ["digraph %s {" % q(self._name), "  compound=true;"]
        for i, g in enumerate(self._groups):
            lines.append("  subgraph %s {" % q("cluster_%d" % i))
            lines.append('    label=%s; style="dashed, rounded";' % q(
                "%d: %s [%s]" % (getattr(g, 'level_time', i), g.name,
                                 g.kind)))
            for c in g.comps:
                live = c.is_output or any(ch not in g.comps
                                          for ch in c.children)
                style = "rounded, bold" if live else "rounded, filled"
                attrs = ['shape=box', 'style="%s"' % style]
                if c in slot:
                    attrs.append('color=%s' % palette[slot[c] %
                                                      len(palette)])
                lines.append("    %s [%s];" % (q(c.func.name),
                                               ", ".join(attrs)))
            lines.append("  }")
        for c in self._comps:
            for pc in c.parents:
                lines.append("  %s -> %s;" % (q(pc.func.name),
                                              q(c.func.name)))
        lines.append("}")
        return PipelineGraph("\n".join(lines) + "\n")

    # ---- code generation and build ----------------------------------------
    def generate_code(self, is_extern_c_func=True, are_io_void_ptrs=True):
        """The CUDA translation unit for this pipeline.  The flags are
        accepted for compatibility; the CUDA target always exports
        ``extern "C"`` entry points taking ``void *`` buffers."""
        from .codegen import generate_code_for_pipeline
        return generate_code_for_pipeline(self)

    def build(self, out_dir=None, verbose=False):
        """Generate, compile (nvcc, sm_100a) and load the pipeline."""
        from .build import build_pipeline
        return build_pipeline(self, out_dir=out_dir, verbose=verbose)


class PipelineGraph(object):
    """Graphviz DOT text of a pipeline's stage graph."""

    def __init__(self, text):
        self._text = text

    def string(self):
        return self._text

    def write(self, path):
        with open(path, "w") as f:
            f.write(self._text)
