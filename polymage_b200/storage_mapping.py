"""Storage mapping of intermediate full arrays in HBM.

The reference keys storage classes on (element size, number of dimensions,
(parameter, coefficient) of each dimension's extent)
(sandbox/storage_mapping.py:114-175) and, under ``optimize_storage``,
reuses an array of the same class once its previous occupant is dead
(:387-435).  Intra-group stages live in tile scratchpads and never reach
this pass; here they live in shared memory or registers (tiling.py).

This backend always reuses: every group live-out that is not a pipeline
output (and is not a const table) gets a slot of its storage class, taken
from the class's free list when a previous occupant's last reader has run.
A slot's byte size is the maximum over its occupants, evaluated per call
from the parameter values, and slots are laid out back to back in one
per-call workspace (256-byte aligned), so the whole pipeline needs one
device allocation that is cached across calls.
"""

from .expression import affine_form
from .liveness import compute_liveness


def storage_key(func):
    dims = []
    for d in func.domain:
        ext = d.upperBound - d.lowerBound + 1
        f = affine_form(ext)
        if f is None:
            dims.append(('?', str(ext)))
        else:
            dims.append(tuple(sorted((k.name, v) for k, v in f[0].items())))
    return (func.typ.size(), len(func.domain), tuple(dims))


def map_storage(pipeline):
    groups = pipeline.groups
    time_of = {}
    for g in groups:
        for c in g.comps:
            time_of[c] = g.level_time
    inter = []
    for g in groups:
        if g.kind == 'const':
            continue
        for comp in g.liveouts():
            if comp.is_output:
                continue
            inter.append(comp)
    children_map = {}
    schedule = {}
    for comp in inter:
        schedule[comp] = time_of[comp]
        kids = [k for k in comp.children if k.group is not comp.group]
        if kids:
            children_map[comp] = kids
    for comp in inter:
        for k in children_map.get(comp, []):
            schedule.setdefault(k, time_of[k])
    liveness = compute_liveness(children_map, schedule)
    last_use = {}
    for t, objs in liveness.items():
        for o in objs:
            last_use[o] = t

    reuse = 'no_storage_reuse' not in pipeline.options
    slots = []            # list of [key, [occupants], free_after_time]
    assign = {}
    for comp in sorted(inter, key=lambda c: time_of[c]):
        key = storage_key(comp.func)
        t = time_of[comp]
        chosen = None
        if reuse:
            for i, s in enumerate(slots):
                if s[0] == key and s[2] < t:
                    chosen = i
                    break
        if chosen is None:
            slots.append([key, [], -1])
            chosen = len(slots) - 1
        slots[chosen][1].append(comp)
        slots[chosen][2] = last_use.get(comp, t)
        assign[comp] = chosen
    pipeline._storage_slots = [s[1] for s in slots]
    pipeline._storage_assign = assign
    return assign
