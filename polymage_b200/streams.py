"""Concurrent launch schedule of a pipeline's groups.

The generated ``pm_run`` launches one kernel (or const-table upload) per
fused group.  Groups that touch disjoint HBM buffers may run at the same
time: the down-sweeps of the two images and the mask of a pyramid blend
are independent chains, and the small launches of its coarse levels leave
most of the GPU idle.  This module assigns every launch to one of a few
CUDA streams and lists the cross-stream event waits that keep every
read-after-write, write-after-read and write-after-write order of the
serial program (HBM buffers include workspace slots that liveness reuses
across groups, so reuse is a write-after-read hazard).  Stream 0 is the
caller's stream; the others fork from it at the start of the call and
join back into it at the end, which stream capture records as a graph
with parallel branches.

The reference runs its groups one after another inside one OpenMP
function (sandbox/codegen.py:920-1067); this schedule has no counterpart
there.
"""


def dependencies(rw):
    """``rw``: per launch, (buffers read, buffers written) as sets.  Returns
    per launch the earlier launches it must follow."""
    deps = []
    for j, (rj, wj) in enumerate(rw):
        d = []
        for i in range(j):
            ri, wi = rw[i]
            if (wi & rj) or (ri & wj) or (wi & wj):
                d.append(i)
        deps.append(d)
    return deps


def schedule(rw, nstreams=4, main_only=()):
    """Stream of every launch and the waits before it.

    Returns (stream_of, waits, records): ``waits[j]`` lists the launches
    whose completion events launch ``j`` waits on (all on other streams),
    ``records`` the launches whose event is recorded after them.  Launches
    in ``main_only`` stay on stream 0.  A launch continues the stream of
    its latest dependency when that stream's last launch is the
    dependency; otherwise it takes a stream whose last launch it depends
    on anyway, or an unused stream, so that no independent work is
    serialized behind it while a stream is free."""
    n = len(rw)
    deps = dependencies(rw)
    main_only = set(main_only)
    last = [-1] * max(1, nstreams)
    stream_of = []
    for j in range(n):
        d = set(deps[j])
        if j in main_only or nstreams <= 1:
            s = 0
        else:
            tails = [k for k in range(nstreams) if last[k] in d]
            free = [k for k in range(nstreams) if last[k] == -1]
            if d and last[stream_of[max(d)]] == max(d):
                s = stream_of[max(d)]
            elif tails:
                s = max(tails, key=lambda k: last[k])
            elif free:
                s = free[0]
            elif d:
                s = stream_of[max(d)]
            else:
                s = min(range(nstreams), key=lambda k: last[k])
        stream_of.append(s)
        last[s] = j
    # waits: per other stream, its latest launch among the dependencies,
    # unless this stream already waited for that one or a later one
    waited = [[-1] * max(1, nstreams) for _ in range(max(1, nstreams))]
    waits = []
    records = set()
    for j in range(n):
        s = stream_of[j]
        need = {}
        for i in deps[j]:
            t = stream_of[i]
            if t != s:
                need[t] = max(need.get(t, -1), i)
        w = []
        for t, i in sorted(need.items()):
            if waited[s][t] >= i:
                continue
            w.append(i)
            records.add(i)
            waited[s][t] = i
        waits.append(w)
    return stream_of, waits, records


def check(rw, stream_of, waits):
    """Whether every dependency is ordered: on the same stream by program
    order, else through a chain of waits (used by the tests)."""
    n = len(rw)
    deps = dependencies(rw)
    # happens-before closure: j follows i if same stream and i < j, or j
    # waited on k with i before k
    before = [set() for _ in range(n)]
    last_on = {}
    for j in range(n):
        s = stream_of[j]
        b = set()
        if s in last_on:
            p = last_on[s]
            b |= before[p] | {p}
        for k in waits[j]:
            b |= before[k] | {k}
        before[j] = b
        last_on[s] = j
    return all(i in before[j] for j in range(n) for i in deps[j])
