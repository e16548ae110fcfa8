"""Automatic grouping of stages for fusion (sandbox/grouping.py:56-239).

The greedy algorithm is the reference's: repeatedly take the first group
that has children and merge it into *all* its children when

  1. the group is not made only of "small" compute objects (a compute
     object is small when its domain has at most ``size_threshold`` points
     while every parent's domain is larger; :73-106),
  2. neither the group nor a child contains a ``Reduction``,
  3. neither contains a ``const`` function,
  4. the merged size stays within ``group_size``, and
  5. with several children, every parent of every child is the group itself
     or one of the children (:186-213);

one merge per iteration until nothing changes.

One extra legality condition comes from the CUDA target: the merged group
must have a valid fused-kernel plan (tiling.py) -- consistent alignment and
scaling, bounded footprints for data-dependent accesses and a shared-memory
footprint within the per-CTA budget.  A merge whose plan fails is skipped
exactly like a merge refused by the criteria above.
"""

import logging

from . import constructs as C
from .bounds import part_boxes
from .evaluate import EvalError

LOG = logging.getLogger("polymage_b200.grouping")


def _comp_sizes(pipeline):
    env = pipeline.int_env()
    sizes = {}
    for comp in pipeline.comps:
        total = 0
        for box, cond, expr, red in part_boxes(comp.func):
            try:
                rng = box.evaluate(env)
            except EvalError:
                total = None
                break
            n = 1
            for lo, hi in rng.values():
                n *= max(0, hi - lo + 1)
            total += n
        sizes[comp] = total
    return sizes


def get_small_comps(pipeline):
    thresh = pipeline._size_threshold
    sizes = _comp_sizes(pipeline)
    small = []
    for comp in pipeline.comps:
        s = sizes[comp]
        is_small = s is not None and s <= thresh
        for p in comp.parents:
            ps = sizes[p]
            if ps is None:
                is_small = False
            else:
                is_small = is_small and ps > thresh
        if is_small:
            small.append(comp)
    return small, sizes


def _plan_ok(pipeline, comps):
    from .tiling import check_group_plan, PlanError
    try:
        check_group_plan(pipeline, comps)
        return True
    except PlanError as e:
        LOG.debug("not merging %s: %s", [c.name for c in comps], e)
        return False


def auto_group(pipeline):
    grp_size = pipeline._group_size
    small, _ = get_small_comps(pipeline)
    small = set(small)
    changed = True
    while changed:
        changed = False
        for group in [g for g in pipeline.groups if g.children]:
            is_small = all(c in small for c in group.comps)
            is_red = any(c.is_reduction for c in group.comps)
            is_const = any(c.is_const_func for c in group.comps)
            for ch in group.children:
                is_red = is_red or any(c.is_reduction for c in ch.comps)
                is_const = is_const or any(c.is_const_func
                                           for c in ch.comps)
            if is_small or is_red or is_const or \
                    len(group.comps) >= grp_size:
                continue
            total = len(group.comps) + sum(len(ch.comps)
                                           for ch in group.children)
            if total > grp_size:
                continue
            if len(group.children) > 1:
                parents_of_children = set()
                for ch in group.children:
                    parents_of_children.update(ch.parents)
                parents_of_children.discard(group)
                if not parents_of_children.issubset(set(group.children)):
                    continue
            merged = list(group.comps)
            for ch in group.children:
                merged += ch.comps
            if not _plan_ok(pipeline, merged):
                continue
            new = group
            for ch in list(group.children):
                new = pipeline.merge_groups(new, ch)
            changed = True
            break


def merge_small(pipeline, limit):
    """Option ('merge_small', N): after the greedy grouping, a group whose
    only child group is C merges into C when every stage of both has at
    most N points (at the parameter estimates) and the merged group has a
    legal plan, whatever the group size.  A single child keeps the merged
    group convex.  Meant for the coarse levels of pyramids, where each
    level's kernel is short and the chain of launches is the cost."""
    _, sizes = get_small_comps(pipeline)

    def small(g):
        return all(sizes.get(c) is not None and sizes[c] <= limit
                   for c in g.comps)

    changed = True
    while changed:
        changed = False
        for group in list(pipeline.groups):
            if len(group.children) != 1:
                continue
            ch = group.children[0]
            if any(c.is_reduction or c.is_const_func
                   for c in group.comps + ch.comps):
                continue
            if not (small(group) and small(ch)):
                continue
            if not _plan_ok(pipeline, list(group.comps) + list(ch.comps)):
                continue
            pipeline.merge_groups(group, ch)
            changed = True
            break


def fuse_all(pipeline):
    """Option 'fuse_all': after the greedy grouping, put every stage that is
    neither a Reduction nor a const function into one group, when that
    group has a legal fused-kernel plan (else the greedy result stands).
    The reference's criterion 5 keeps a DAG like the camera pipe's
    demosaic (stages read by several siblings) in many groups, each
    writing its planes to memory and reading them back; one overlapped
    tile over the whole DAG recomputes halos instead."""
    groups = [g for g in pipeline.groups
              if not any(c.is_reduction or c.is_const_func for c in g.comps)]
    if len(groups) < 2:
        return
    merged = []
    for g in groups:
        merged += g.comps
    if not _plan_ok(pipeline, merged):
        return
    # merge in an order that keeps every intermediate group convex: the
    # groups are merged into the first one following the schedule order
    new = groups[0]
    for g in groups[1:]:
        new = pipeline.merge_groups(new, g)


def manual_group(pipeline, grouping):
    """User-specified grouping: a list of lists of Functions (the original
    objects passed to buildPipeline).  Functions not listed stay alone, and
    so does a Function given directly as an entry (the reference's tests
    also pass a flat list: sandbox/tests/test_stencil.py:58)."""
    for funcs in grouping:
        if not isinstance(funcs, (list, tuple)):
            funcs = [funcs]
        comps = []
        for f in funcs:
            clone = pipeline._clone_map.get(f, f)
            if clone not in pipeline.func_map:
                raise ValueError("grouping names %s, which is not in the "
                                 "pipeline" % getattr(f, 'name', f))
            comps.append(pipeline.func_map[clone])
        groups = []
        for c in comps:
            if c.group not in groups:
                groups.append(c.group)
        if len(groups) < 2:
            continue
        merged = []
        for g in groups:
            merged += g.comps
        from .tiling import check_group_plan
        check_group_plan(pipeline, merged)
        new = groups[0]
        for g in groups[1:]:
            new = pipeline.merge_groups(new, g)
