"""Concurrent launch schedule (no GPU): every read-after-write,
write-after-read and write-after-write order of the serial program is kept
by stream order or by event waits, on random buffer sets and on the
shipped pipelines' groups."""

import numpy as np
import pytest

from polymage_b200 import streams
from polymage_b200.apps import catalog
from polymage_b200.codegen import PipelineGen


def _random_rw(rng, n, nbuf):
    rw = []
    for _ in range(n):
        r = set(rng.integers(0, nbuf, rng.integers(0, 4)).tolist())
        w = set(rng.integers(0, nbuf, rng.integers(0, 3)).tolist())
        rw.append((r, w))
    return rw


@pytest.mark.parametrize("nstreams", [1, 2, 3, 4, 6])
def test_random_programs_keep_every_order(nstreams):
    rng = np.random.default_rng(nstreams)
    for _ in range(300):
        rw = _random_rw(rng, int(rng.integers(1, 30)), int(rng.integers(1,
                                                                         12)))
        sof, waits, records = streams.schedule(rw, nstreams)
        assert streams.check(rw, sof, waits)
        assert all(0 <= s < nstreams for s in sof)
        assert all(i in records for w in waits for i in w)
        for j, w in enumerate(waits):
            assert all(i < j and sof[i] != sof[j] for i in w)


def test_independent_chains_use_separate_streams():
    # three chains a0->a1, b0->b1, c0->c1 interleaved, then a join
    rw = [({'x'}, {'a0'}), ({'x'}, {'b0'}), ({'x'}, {'c0'}),
          ({'a0'}, {'a1'}), ({'b0'}, {'b1'}), ({'c0'}, {'c1'}),
          ({'a1', 'b1', 'c1'}, {'out'})]
    sof, waits, _ = streams.schedule(rw, 4)
    assert len(set(sof[:3])) == 3
    assert sof[3] == sof[0] and sof[4] == sof[1] and sof[5] == sof[2]
    assert len(waits[6]) == 2 and streams.check(rw, sof, waits)


def test_workspace_reuse_is_a_hazard():
    # launch 2 reuses the slot that launch 1 reads: it must wait for it
    rw = [({'in'}, {'slot0'}), ({'slot0'}, {'out1'}), ({'in'}, {'slot0'})]
    sof, waits, _ = streams.schedule(rw, 4)
    assert streams.check(rw, sof, waits)


def test_main_only_launches_stay_on_the_callers_stream():
    rw = [({'x'}, {'a'}), ({'x'}, {'t'}), ({'t', 'a'}, {'o'})]
    sof, _, _ = streams.schedule(rw, 4, main_only=[1])
    assert sof[1] == 0


@pytest.mark.parametrize("name", ["pyramid", "campipe", "bilateral"])
def test_shipped_pipelines_schedule(name):
    b, kw = catalog._BUILDERS[name]
    p = b(**kw)
    mod = p.generate_code()
    pg = PipelineGen(p)
    pg.slot_of = getattr(p, '_storage_assign', {})
    rw = [pg.group_rw(g) for g in p.groups]
    sof, waits, _ = streams.schedule(rw, 4)
    assert streams.check(rw, sof, waits)
    if name == "pyramid":
        # the down-sweeps of img1, img2 and the mask are independent
        assert len(set(sof)) == 3
        assert "pm_conc_get" in mod.source


def test_checker_catches_a_missing_wait():
    rw = [({'x'}, {'a0'}), ({'x'}, {'b0'}), ({'a0', 'b0'}, {'out'})]
    sof, waits, _ = streams.schedule(rw, 4)
    assert streams.check(rw, sof, waits) and waits[2]
    assert not streams.check(rw, sof, [[], [], []])


@pytest.mark.parametrize("name", ["laplacian", "pyramid8", "vcycle",
                                  "wcycle", "nas_mg", "interpolate"])
def test_schedules_of_larger_pipelines_keep_every_order(name):
    """Deeper DAGs with workspace slots reused across many groups."""
    if name in ("laplacian", "pyramid8"):
        b, kw = catalog._BUILDERS[name]
        p = b(**kw)
    elif name == "vcycle":
        from polymage_b200.apps.multigrid import build_v_cycle
        p = build_v_cycle(n=63, L=3)
    elif name == "wcycle":
        from polymage_b200.apps.multigrid import build_v_cycle
        p = build_v_cycle(n=63, L=3, gamma=2, name="Wcycle")
    elif name == "nas_mg":
        from polymage_b200.apps.nas_mg import build_mg3p
        p = build_mg3p('S')
    else:
        from polymage_b200.apps.interpolate import build_interpolate
        p = build_interpolate(rows=512, cols=512)
    p.generate_code()
    pg = PipelineGen(p)
    pg.slot_of = getattr(p, '_storage_assign', {})
    rw = [pg.group_rw(g) for g in p.groups]
    for nst in (2, 3, 4):
        sof, waits, _ = streams.schedule(rw, nst)
        assert streams.check(rw, sof, waits)
