"""What the trained cost model gains over tuning without it.

Replays the learned tuner on the committed B200 timing database (every
configuration of the reference's search space, measured): for each pipeline
the model is pretrained on the *other* pipelines only (on the GPU, by this
package's kernels) and picks 8 configurations, which are then "timed" by
looking them up.  Without the model, the same budget of 8 timed
configurations is spent on a random choice."""

import numpy as np
import pytest

from polymage_b200 import costmodel, tuner

pytestmark = pytest.mark.gpu


def test_learned_beats_random_budget_and_reaches_near_best(cuda):
    rows = tuner.load_db(costmodel.DB_PATH)
    apps = sorted(set(r['app'] for r in rows))
    assert len(apps) >= 5
    learned, random6 = [], []
    for app in apps:
        ratio, n, uniq = costmodel.evaluate_on_db(rows, app, batches=(8,),
                                                  seed=0)
        assert n == 8
        learned.append(ratio)
        ms = {}
        for r in rows:
            if r['app'] == app:
                k = costmodel.signature(r['features'], r)
                ms[k] = min(ms.get(k, 1e9), r['ms'])
        v = np.array(list(ms.values()))
        rnd = np.mean([np.random.default_rng(s).choice(v, 8, replace=False)
                       .min() / v.min() for s in range(300)])
        random6.append(rnd)
        print(app, "learned %.3f random %.3f (distinct plans %d)" % (
            ratio, rnd, uniq))
    assert np.mean(learned) < np.mean(random6)
    assert np.mean(learned) <= 1.10
    assert sum(r <= 1.05 for r in learned) >= 3
