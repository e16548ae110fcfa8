"""Liveness of compute objects under a schedule (sandbox/liveness.py:35-88).

``compute_liveness(children_map, schedule)`` maps each schedule time to the
objects whose last consumer runs at that time; objects without children
never die.  The pipeline applies it to groups' live-outs to decide when an
intermediate HBM buffer can be reused by a later group (storage_mapping.py).
"""


def compute_liveness(children_map, schedule):
    liveness_map = {}
    for obj in schedule:
        if obj not in children_map:
            continue
        last = -1
        for child in children_map[obj]:
            last = max(last, schedule[child])
        liveness_map.setdefault(last, []).append(obj)
    return liveness_map


def liveness_for_pipe_outputs(pipeline):
    """Liveness of every group live-out, keyed by group schedule time."""
    schedule = {}
    children = {}
    for g in pipeline.groups:
        for comp in g.liveouts():
            schedule[comp] = g.level_time
            kids = [ch for ch in comp.children if ch.group is not g]
            if kids:
                children[comp] = kids
    # a child's time is its group's time
    child_sched = dict(schedule)
    for g in pipeline.groups:
        for c in g.comps:
            child_sched.setdefault(c, g.level_time)
    lmap = {}
    for comp, kids in children.items():
        last = max(child_sched[k] for k in kids)
        lmap.setdefault(last, []).append(comp)
    pipeline._liveness_map = lmap
    return lmap
