"""Chain planning (option ``chain``) on CPU: which groups share a launch,
the phase order inside it, and the generated kernel's shape.  A member
that reads a function another member writes runs in a later phase; members
are consecutive launches of one CTA size; the per-group kernels stay for
the batched entries."""

import pytest

from polymage_b200.apps import catalog
from polymage_b200.pipe import body_refs


def _chains(name, opts=('chain',)):
    p = catalog.variant(name, opts)
    mod = p.generate_code()
    return p, mod


def _groups_by_kernel(p):
    out = {}
    for g in p.groups:
        out["pm_%s_g%d" % (p.name, g.level_time)] = g
    return out


@pytest.mark.parametrize("name", ["vcycle", "wcycle", "pyramid8",
                                  "interpolate", "laplacian"])
def test_chain_phases_follow_dependences(name):
    p, mod = _chains(name)
    chains = mod.meta.get('chains')
    assert chains, "no chain formed"
    by_k = _groups_by_kernel(p)
    order = [("pm_%s_g%d" % (p.name, g.level_time)) for g in p.groups]
    for ch in chains:
        idx = [order.index(k) for k in ch['members']]
        assert idx == list(range(idx[0], idx[0] + len(idx))), \
            "members are not consecutive launches"
        assert all(by_k[k].plan.kind == 'stencil' for k in ch['members'])
        assert len(set(by_k[k].plan.threads for k in ch['members'])) == 1
        ph = dict(zip(ch['members'], ch['phases']))
        writes = dict((k, set(id(c.func) for c in by_k[k].comps))
                      for k in ch['members'])
        for j in ch['members']:
            reads = set(id(r.objectRef) for c in by_k[j].comps
                        for r in body_refs(c.func))
            for i in ch['members']:
                if order.index(i) < order.index(j) and writes[i] & reads:
                    assert ph[i] < ph[j], (i, j, ph[i], ph[j])
        assert "%s_body<true>" % ch['members'][0] in mod.source
    ngroups = sum({'stencil': 1, 'reduction': 2}.get(g.plan.kind, 0)
                  for g in p.groups)
    assert mod.meta['launches'] == ngroups - sum(
        len(c['members']) - 1 for c in chains)
    # the batched entries keep one launch per group
    for k in by_k:
        if by_k[k].plan.kind == 'stencil':
            assert "batch_%s(" % k in mod.source


def test_no_chain_without_the_option():
    p, mod = _chains("vcycle", ())
    assert not mod.meta.get('chains')
    assert "pm_grid_sync" not in mod.source.split("#include")[-1]


def test_chain_limit_and_independent_members():
    """With a limit of 64 tiles the 8-level pyramid chains only its coarse
    levels; the down-sweeps of the two images and the mask share phases."""
    p, mod = _chains("pyramid8", (('chain', 64),))
    chains = mod.meta['chains']
    by_k = _groups_by_kernel(p)
    from polymage_b200.grouping import _comp_sizes
    import numpy as np
    sizes = _comp_sizes(p)
    for ch in chains:
        for k in ch['members']:
            plan = by_k[k].plan
            assert sizes[p.func_map[plan.anchor]] / np.prod(plan.tile) <= 64
        assert max(ch['phases']) + 1 < len(ch['members'])


def test_chain_barrier_is_bounded():
    """The grid barrier gives up after a bounded number of polls and
    records the timeout in the error word."""
    import os
    from polymage_b200.build import CSRC
    src = open(os.path.join(CSRC, "pm_runtime.cuh")).read()
    body = src[src.index("bool pm_grid_sync"):]
    body = body[:body.index("\n}\n")]
    assert "PM_GRID_WAIT_LIMIT" in body and "PM_KERR_GRID_TIMEOUT" in body
