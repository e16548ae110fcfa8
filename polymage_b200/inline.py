"""Inline pass: substitute user-listed functions into their consumers
(sandbox/inline.py:29-199).

The reference inlines a directive's function when every use reads values
produced by one predicate-free piece of its definition.  This backend
inlines functions whose definition is a single expression, and those
defined by a single ``Case(cond, e)``, which become ``Select(cond, e, 0)``
at each use: the value of a point the Case does not cover is 0, the
convention for uncomputed points, so the substitution is exact whether or
not the reads stay inside the Case.  Piecewise definitions are kept, with
a warning.  Independently
of directives, the CUDA code generator computes cheap pointwise stages in
registers at their use points (tiling.py), which is where most of the
reference's explicit inlining benefit comes from on a GPU.
"""

import logging

from . import constructs as C
from .expr_ast import Value
from .expression import rebuild, rebuild_cond, substitute_vars

LOG = logging.getLogger("polymage_b200.inline")


def _single_expression(func):
    d = func.defn
    return len(d) == 1 and not isinstance(d[0], (C.Case, C.Reduce))


def _single_case(func):
    d = func.defn
    return len(d) == 1 and isinstance(d[0], C.Case) and \
        not isinstance(d[0].expression, C.Reduce)


def inline_pass(pipeline):
    for directive in pipeline._inline_directives:
        clone = pipeline._clone_map.get(directive)
        if clone is None or clone not in pipeline.func_map:
            LOG.warning("inline directive %s is not in the pipeline",
                        getattr(directive, 'name', directive))
            continue
        comp = pipeline.func_map[clone]
        if comp.is_output or isinstance(clone, C.Reduction) or \
                clone.is_const_func:
            LOG.warning("cannot inline %s (output, reduction or const)",
                        clone.name)
            continue
        if _single_expression(clone):
            body = clone.defn[0]
        elif _single_case(clone):
            case = clone.defn[0]
            body = C.Select(case.condition, case.expression,
                            Value(0, clone.typ), typeCheck=False)
        else:
            LOG.warning("not inlining %s: piecewise definitions are kept",
                        clone.name)
            continue

        def leaf(n, clone=clone, body=body):
            if isinstance(n, C.Reference) and n.objectRef is clone:
                args = [rebuild(a, leaf) for a in n.arguments]
                return substitute_vars(body, dict(zip(clone.variables,
                                                      args)))
            return None

        for child in list(comp.children):
            f = child.func
            parts = []
            for p in f.defn:
                if isinstance(p, C.Case):
                    e = p.expression
                    if isinstance(e, C.Reduce):
                        e = C.Reduce(rebuild(e.accumulate_ref, leaf),
                                     rebuild(e.expression, leaf), e.op_type)
                    else:
                        e = rebuild(e, leaf)
                    parts.append(C.Case(rebuild_cond(p.condition, leaf), e))
                elif isinstance(p, C.Reduce):
                    parts.append(C.Reduce(rebuild(p.accumulate_ref, leaf),
                                          rebuild(p.expression, leaf),
                                          p.op_type))
                else:
                    parts.append(rebuild(p, leaf))
            f._body = parts
            # rewire: the child now reads the inlined function's parents
            child.parents = [p for p in child.parents if p is not comp]
            for gp in comp.parents:
                if gp not in child.parents:
                    child.parents.append(gp)
                if child not in gp.children:
                    gp.children.append(child)
            for im in comp.images:
                if all(im is not q for q in child.images):
                    child.images.append(im)
        pipeline.drop_comp(comp)
