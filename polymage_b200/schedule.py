"""Ordering of groups and of compute objects inside a group.

Groups run level by level in a topological order (sandbox/schedule.py:85,
``level_order`` sandbox/utils.py:120-138); inside a group, compute objects
run in topological order (sandbox/schedule.py:128).  Each group gets a
``level_time`` (its position in the launch sequence) used by liveness.
"""


def level_order(objs, parent_map):
    """Topological level of every object: 0 for objects without parents,
    else one more than the deepest parent (sandbox/utils.py:120-138)."""
    order = dict((o, 0) for o in objs)
    changed = True
    while changed:
        changed = False
        for o in objs:
            for p in parent_map.get(o) or []:
                if p in order and order[p] >= order[o]:
                    order[o] = order[p] + 1
                    changed = True
    return order


def schedule_groups(pipeline):
    groups = pipeline.groups
    parent_map = dict((g, list(g.parents)) for g in groups)
    levels = level_order(groups, parent_map)
    # stable order: by level, then by the position of the group's first
    # compute object in the pipeline's topological order
    pos = dict((c, i) for i, c in enumerate(pipeline.comps))
    groups.sort(key=lambda g: (levels[g], min(pos[c] for c in g.comps)))
    for t, g in enumerate(groups):
        g.level = levels[g]
        g.level_time = t
        g.comps.sort(key=lambda c: pos[c])
    pipeline._groups = groups
