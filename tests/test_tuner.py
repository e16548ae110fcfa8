"""Tuner generate step, timing database and cost-model features (no GPU)."""

import json
import os

import numpy as np

from polymage_b200 import tuner
from polymage_b200.autotune import app_setup
from polymage_b200.costmodel import featurize, FEATURES, relative_targets


def test_generate_small_space(tmp_path):
    a = app_setup('harris')
    a['_tuner_tile_size_configs'] = [[32, 64], [16, 128]]
    a['_tuner_group_size_configs'] = [3, 11]
    a['_tuner_dst_path'] = str(tmp_path)
    a['_tuner_jobs'] = 4
    src, n, pipe = tuner.generate(a)
    assert n == 4 and pipe is not None
    man = json.load(open(os.path.join(src, "configurations.json")))
    assert [c['status'] for c in man['configs']] == ['built'] * 4
    for c in man['configs']:
        assert os.path.exists(c['so'])
        assert c['features']['ngroups'] >= 1
        x = featurize(c['features'], c, 2048 * 2048)
        assert x.shape == (len(FEATURES),) and np.all(np.isfinite(x))


def test_plan_failure_is_skipped(tmp_path):
    a = app_setup('unsharp')
    # a tile too large for shared memory: the plan fails, the tuner goes on
    a['_tuner_tile_size_configs'] = [[256, 256], [32, 128]]
    a['_tuner_group_size_configs'] = [11]
    a['_tuner_dst_path'] = str(tmp_path)
    src, n, pipe = tuner.generate(a)
    man = json.load(open(os.path.join(src, "configurations.json")))
    st = [c['status'] for c in man['configs']]
    assert st[0] in ('plan_failed', 'built') and st[1] == 'built'


def test_timing_db_roundtrip_and_torn_line(tmp_path):
    db = str(tmp_path / "db.jsonl")
    e = {'key': 'k1', 'tile': [32, 64], 'group_size': 5, 'options': [],
         'features': {'ngroups': 1}}
    tuner.record(db, 'harris', e, 0.5, '[["img", [64, 64]]]')
    tuner.record(db, 'harris', dict(e, key='k2'), 0.25, '[["img", [64, 64]]]')
    with open(db, "a") as f:
        f.write('{"app": "harris", "ms": ')     # torn by a crash
    rows = tuner.load_db(db)
    assert len(rows) == 2
    t = relative_targets(rows)
    assert abs(t.sum()) < 1e-6 and t[0] > t[1]


def test_measure_option_parsing_matches_catalog_options():
    """measure --options / --drop-options: nested JSON lists become the
    nested tuples the catalog writes, so a catalog option can be left out
    by restating it."""
    from polymage_b200.apps import catalog
    from polymage_b200.apps.measure import parse_options
    order = [o for o in catalog.MAXFILTER['options']
             if isinstance(o, tuple) and o[0] == 'storage_order']
    text = '[["storage_order",[["vert",[3,0,1,2]],["vert_log",[3,0,1,2]]]]]'
    assert parse_options(text) == order
    assert parse_options(None) == []
    assert parse_options('["chain", "rblock=4"]') == ['chain', 'rblock=4']
    p = catalog.variant("maxfilter", (), parse_options(text))
    assert not any(isinstance(o, tuple) and o[0] == 'storage_order'
                   for o in p.options)
