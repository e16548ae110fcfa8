"""Learned cost model for the tuner.

A small MLP (FP32, three hidden layers of 128, ReLU) maps the plan
features of a pipeline configuration (group structure, tile sizes, halo,
shared-memory bytes, threads, recompute cost ... -- ``tuner.
pipeline_features``) to its log kernel time relative to the other
configurations of the same pipeline and input.  It is trained on the GPU by
the hand-written kernels of ``csrc/mlp.cu`` (forward, backward, Adam) on the
measurements the tuner appends to its timing database, and ranks
configurations so that only the top-k are compiled and timed
(``learned_tune``); the exhaustive tuner stays as the fallback and as the
measure of the ranking's error.
"""

import ctypes
import json
import math
import os
import time

import numpy as np

from .build import compile_source, GEN_DIR, CSRC

FEATURES = ['ngroups', 'nstencil', 'nred', 'stages', 'smem_max', 'smem_sum',
            'halo_max', 'redund_sum', 'tile_inner', 'tile_outer', 'threads',
            'cost_sum', 'nsmem', 'nstage_in', 'ninline', 'group_size',
            'tile0', 'tile1', 'rblock', 'log_pixels']
HIDDEN = 128

_lib = None


def lib():
    """The cost model's CUDA library (built in-tree on first use)."""
    global _lib
    if _lib is None:
        so = compile_source("mlp", os.path.join(CSRC, "mlp.cu"))
        L = ctypes.CDLL(so)
        L.pm_mlp_param_count.restype = ctypes.c_long
        L.pm_mlp_param_count.argtypes = [ctypes.c_int, ctypes.c_int]
        L.pm_mlp_act_count.restype = ctypes.c_long
        L.pm_mlp_act_count.argtypes = [ctypes.c_int, ctypes.c_int]
        L.pm_mlp_work_count.restype = ctypes.c_long
        L.pm_mlp_work_count.argtypes = [ctypes.c_int, ctypes.c_int]
        L.pm_mlp_forward.argtypes = [ctypes.c_void_p, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_void_p,
                                     ctypes.c_int, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_void_p]
        L.pm_mlp_backward.argtypes = [ctypes.c_void_p, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_int] + \
            [ctypes.c_void_p] * 5
        L.pm_mlp_adam.argtypes = [ctypes.c_void_p] * 4 + \
            [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
             ctypes.c_float, ctypes.c_void_p]
        _lib = L
    return _lib


def featurize(features, cfg, pixels):
    """Feature vector (log-scaled) of one configuration."""
    f = dict(features)
    tile = list(cfg['tile'])
    f['group_size'] = cfg['group_size']
    f['tile0'] = tile[-2] if len(tile) > 1 else 1
    f['tile1'] = tile[-1]
    rb = 4
    for o in cfg.get('options', []):
        if isinstance(o, str) and o.startswith('rblock='):
            rb = int(o.split('=')[1])
    f['rblock'] = rb
    f['log_pixels'] = math.log(max(pixels, 1))
    return np.array([math.log1p(max(float(f.get(k, 0.0)), 0.0))
                     for k in FEATURES], np.float32)


def pixels_of(data_key):
    """Pixel count of a timing-database row's input (largest array)."""
    try:
        shapes = json.loads(data_key)
    except ValueError:
        return 1
    best = 1
    for _, s in shapes:
        n = 1
        for d in s[-2:]:
            n *= d
        best = max(best, n)
    return best


def relative_targets(rows):
    """log(ms) minus the mean log(ms) of the row's (app, input) group."""
    groups = {}
    for r in rows:
        groups.setdefault((r['app'], r['data']), []).append(math.log(r['ms']))
    means = dict((k, sum(v) / len(v)) for k, v in groups.items())
    return np.array([math.log(r['ms']) - means[(r['app'], r['data'])]
                     for r in rows], np.float32)


class CostModel(object):
    def __init__(self, D=len(FEATURES), H=HIDDEN, seed=0):
        import torch
        self.D, self.H = D, H
        L = lib()
        n = L.pm_mlp_param_count(D, H)
        rng = np.random.default_rng(seed)
        p = np.zeros(n, np.float32)
        # He initialization per layer
        o = 0
        for fan_in, fan_out in ((D, H), (H, H), (H, H), (H, 1)):
            w = rng.normal(0, math.sqrt(2.0 / fan_in), fan_out * fan_in)
            p[o:o + w.size] = w
            o += w.size + fan_out
        self.dev = torch.device('cuda', torch.cuda.current_device())
        self.params = torch.from_numpy(p).to(self.dev)
        self.mu = np.zeros(D, np.float32)
        self.sd = np.ones(D, np.float32)
        self.history = []

    def _x(self, X):
        import torch
        Xn = (np.asarray(X, np.float32) - self.mu) / self.sd
        return torch.from_numpy(np.ascontiguousarray(Xn)).to(self.dev)

    def fit(self, X, y, epochs=600, lr=2e-3, weight_decay=1e-4):
        """Full-batch Adam on the GPU; returns the loss curve."""
        import torch
        X = np.asarray(X, np.float32)
        self.mu = X.mean(0)
        self.sd = X.std(0) + 1e-3
        L = lib()
        B = X.shape[0]
        xd = self._x(X)
        yd = torch.from_numpy(np.asarray(y, np.float32)).to(self.dev)
        acts = torch.zeros(L.pm_mlp_act_count(B, self.H), device=self.dev)
        work = torch.zeros(L.pm_mlp_work_count(B, self.H), device=self.dev)
        grads = torch.zeros_like(self.params)
        m = torch.zeros_like(self.params)
        v = torch.zeros_like(self.params)
        loss = torch.zeros(1, device=self.dev)
        s = torch.cuda.current_stream().cuda_stream
        losses = []
        for t in range(1, epochs + 1):
            st = L.pm_mlp_backward(self.params.data_ptr(), self.D, self.H,
                                   xd.data_ptr(), yd.data_ptr(), B,
                                   acts.data_ptr(), work.data_ptr(),
                                   grads.data_ptr(), loss.data_ptr(), s)
            st |= L.pm_mlp_adam(self.params.data_ptr(), grads.data_ptr(),
                                m.data_ptr(), v.data_ptr(), self.D, self.H,
                                t, lr, weight_decay, s)
            if st:
                raise RuntimeError("cost model kernels failed")
            if t % 50 == 0 or t == 1:
                losses.append(float(loss.item()))
        self.history = losses
        return losses

    def predict(self, X):
        import torch
        L = lib()
        X = np.asarray(X, np.float32)
        B = X.shape[0]
        xd = self._x(X)
        acts = torch.zeros(L.pm_mlp_act_count(B, self.H), device=self.dev)
        out = torch.zeros(B, device=self.dev)
        st = L.pm_mlp_forward(self.params.data_ptr(), self.D, self.H,
                              xd.data_ptr(), B, acts.data_ptr(),
                              out.data_ptr(),
                              torch.cuda.current_stream().cuda_stream)
        if st:
            raise RuntimeError("cost model forward failed")
        return out.cpu().numpy()

    def save(self, path):
        np.savez(path, params=self.params.cpu().numpy(), mu=self.mu,
                 sd=self.sd, D=self.D, H=self.H)

    @classmethod
    def load(cls, path):
        import torch
        z = np.load(path)
        m = cls(int(z['D']), int(z['H']))
        m.params = torch.from_numpy(z['params']).to(m.dev)
        m.mu, m.sd = z['mu'], z['sd']
        return m


def train_from_rows(rows, exclude_app=None, epochs=600, seed=0):
    rows = [r for r in rows if r['app'] != exclude_app]
    X = np.stack([featurize(r['features'], r, pixels_of(r['data']))
                  for r in rows])
    y = relative_targets(rows)
    model = CostModel(seed=seed)
    model.fit(X, y, epochs=epochs)
    return model


DB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                       "timing_db_b200.jsonl")


def signature(features, cfg):
    """Configurations with equal signatures generate the same code."""
    return json.dumps([sorted(features.items()), list(cfg['tile']),
                       [list(o) if isinstance(o, tuple) else o
                        for o in cfg.get('options', [])]])


def app_normalized(X, groups):
    """Features minus their mean over the configurations of the same
    pipeline and input (the targets are relative to that group too)."""
    X = np.array(X, np.float32)
    out = X.copy()
    for g in set(groups):
        idx = [i for i, h in enumerate(groups) if h == g]
        out[idx] = X[idx] - X[idx].mean(0)
    return out


def db_training_set(rows, exclude_app=None):
    """(X, y) of the timing database, one row per distinct plan, features
    and targets relative to each (pipeline, input) group."""
    uniq = {}
    for r in rows:
        if r['app'] == exclude_app:
            continue
        k = (r['app'], r['data'], signature(r['features'], r))
        if k not in uniq or r['ms'] < uniq[k]['ms']:
            uniq[k] = r
    rs = list(uniq.values())
    if not rs:
        return np.zeros((0, len(FEATURES)), np.float32), np.zeros(0,
                                                                   np.float32)
    X = np.stack([featurize(r['features'], r, pixels_of(r['data']))
                  for r in rs])
    X = app_normalized(X, [(r['app'], r['data']) for r in rs])
    return X, relative_targets(rs)


def _plan_worker(job):
    app, cfg = job
    from .autotune import app_setup
    from . import tuner
    try:
        p = tuner.plan_config(app_setup(app), cfg, app)
        return tuner.pipeline_features(p)
    except Exception:
        return None


def plan_candidates(arg_data, configs, jobs=None, app_for_workers=None):
    """Plan features of every configuration (None for plans that fail).
    Shipped pipelines are planned in parallel worker processes (spawned:
    the workers rebuild the spec by name); others sequentially."""
    import sys
    from . import tuner
    name = arg_data.get('_tuner_pipe_name') or arg_data['_tuner_app_name']

    def one(cfg):
        try:
            return tuner.pipeline_features(
                tuner.plan_config(arg_data, cfg, name))
        except Exception:
            return None

    if not configs:
        return []
    # the first plan, timed: a pool pays off only when planning them all
    # one after another would take longer than starting its workers
    t0 = time.time()
    first = one(configs[0])
    serial_s = (time.time() - t0) * len(configs)
    main_file = getattr(sys.modules.get('__main__'), '__file__', None)
    spawnable = main_file is not None and os.path.exists(main_file)
    if app_for_workers is not None and len(configs) > 8 and spawnable and \
            serial_s > 4.0:
        import multiprocessing as mp
        jobs = jobs or max(1, (os.cpu_count() or 2) - 1)
        ctx = mp.get_context("spawn")
        pool = ctx.Pool(jobs)
        try:
            res = pool.map_async(_plan_worker,
                                 [(app_for_workers, c) for c in configs[1:]],
                                 chunksize=max(1, len(configs) //
                                               (4 * jobs)))
            return [first] + res.get(timeout=600)
        finally:
            pool.terminate()
            pool.join()
    return [first] + [one(cfg) for cfg in configs[1:]]


def _rblock(cfg):
    for o in cfg.get('options', []):
        if isinstance(o, str) and o.startswith('rblock='):
            return int(o.split('=')[1])
    return 4


def neighbours(a, b):
    """True when configuration ``a`` differs from ``b`` by one step of one
    knob: a tile side halved or doubled, the register blocking, or the
    group size."""
    ta, tb = a['tile'], b['tile']
    steps = 0
    for x, y in ((ta[-2] if len(ta) > 1 else 1, tb[-2] if len(tb) > 1
                  else 1), (ta[-1], tb[-1])):
        if x != y:
            steps += 1 if x in (2 * y, y // 2) else 9
    if _rblock(a) != _rblock(b):
        steps += 1
    if a['group_size'] != b['group_size']:
        steps += 1
    return steps == 1


class OnlineRanker(object):
    """The online protocol shared by the live tuner and its replay on
    recorded timings: an ensemble of cost models pretrained on other
    pipelines' measurements, retrained on the GPU after every batch with
    this pipeline's own measurements (weighted ``repeat`` times)."""

    def __init__(self, Xc, Xb, yb, ensemble=3, epochs=200, repeat=20,
                 seed=0):
        self.Xc, self.Xb, self.yb = Xc, Xb, yb
        self.ensemble, self.epochs, self.repeat = ensemble, epochs, repeat
        self.seed = seed
        self.measured = {}

    def order(self):
        idx = [i for i, ms in self.measured.items() if ms is not None]
        X, y = self.Xb, self.yb
        if len(idx) >= 2:
            ym = np.log([self.measured[i] for i in idx])
            ym = (ym - ym.mean()).astype(np.float32)
            X = np.concatenate([self.Xb] + [self.Xc[idx]] * self.repeat)
            y = np.concatenate([self.yb] + [ym] * self.repeat)
        if len(X) == 0:
            return list(range(len(self.Xc)))
        pred = np.zeros(len(self.Xc), np.float32)
        for e in range(self.ensemble):
            m = CostModel(seed=self.seed * 100 + len(self.measured) * 7 + e)
            m.fit(X, y, epochs=self.epochs)
            pred += m.predict(self.Xc)
        return [int(i) for i in np.argsort(pred)]

    def run(self, cands, measure, batches=(8,), local=0):
        for b in batches:
            pick = [i for i in self.order() if i not in self.measured][:b]
            if not pick:
                break
            for i, ms in zip(pick, measure(pick)):
                self.measured[i] = ms
        ok = [i for i, ms in self.measured.items() if ms is not None]
        if ok and local:
            bi = min(ok, key=lambda i: self.measured[i])
            pick = [i for i in self.order() if i not in self.measured and
                    neighbours(cands[i], cands[bi])][:local]
            for i, ms in zip(pick, measure(pick) if pick else []):
                self.measured[i] = ms
        ok = [i for i, ms in self.measured.items() if ms is not None]
        return min(ok, key=lambda i: self.measured[i]) if ok else None


def learned_tune(arg_data, db_rows=None, batches=(8,), local=0,
                 ensemble=3, seed=0, shipped_app=None, measure=None):
    """Online learned tuning of one pipeline: plan every configuration of
    the search space (no compilation), keep one per distinct plan, then
    time only what the cost model ranks first (``OnlineRanker.run``).
    ``measure(configs)`` returns their times in ms (default: compile with
    ``tuner.generate`` and time with ``tuner.execute``).  Returns a dict
    with the best configuration, every measurement and the wall-clock
    seconds spent, planning included."""
    from . import tuner
    t0 = time.time()
    a = dict(arg_data)
    app = a['_tuner_app_name']
    configs = a.get('_tuner_configs') or tuner.enumerate_configs(
        a.get('_tuner_tile_size_configs') or tuner.DEFAULT_TILES,
        a.get('_tuner_group_size_configs') or tuner.DEFAULT_GROUPS,
        a.get('_tuner_option_configs'))
    feats = plan_candidates(a, configs, app_for_workers=shipped_app)
    pix = pixels_of(tuner.data_key(a['_tuner_pipe_arg_data']))
    cands, cfeat, seen = [], [], set()
    for cfg, f in zip(configs, feats):
        if f is None:
            continue
        s = signature(f, cfg)
        if s in seen:
            continue
        seen.add(s)
        cands.append(cfg)
        cfeat.append(featurize(f, cfg, pix))
    Xc = app_normalized(np.stack(cfeat), [0] * len(cands))
    if db_rows is None:
        db_rows = tuner.load_db(DB_PATH)
    Xb, yb = db_training_set(db_rows, exclude_app=app)
    t_plan = time.time() - t0

    spent = {'compile_s': 0.0, 'time_s': 0.0}

    def default_measure(idx):
        b = dict(a)
        b['_tuner_configs'] = [cands[i] for i in idx]
        t1 = time.time()
        src, n, pipe = tuner.generate(b)
        t2 = time.time()
        b['_tuner_src_path'] = src
        b['_tuner_pipe'] = pipe
        rep = tuner.execute(b)
        spent['compile_s'] += t2 - t1
        spent['time_s'] += time.time() - t2
        got = dict((json.dumps([r['tile'], r['group_size'], r['options']]),
                    r['ms']) for r in rep['results'])
        return [got.get(json.dumps([cands[i]['tile'], cands[i]['group_size'],
                                    cands[i]['options']])) for i in idx]

    meas = (lambda idx: measure([cands[i] for i in idx])) if measure \
        else default_measure
    ranker = OnlineRanker(Xc, Xb, yb, ensemble=ensemble, seed=seed)
    best = ranker.run(cands, meas, batches=batches, local=local)
    return {'app': app,
            'best': cands[best] if best is not None else None,
            'best_ms': ranker.measured[best] if best is not None else None,
            'measured': [{'config': cands[i], 'ms': ms}
                         for i, ms in ranker.measured.items()],
            'candidates': len(cands), 'plan_s': t_plan,
            'compile_s': spent['compile_s'], 'time_s': spent['time_s'],
            'wall_s': time.time() - t0}


def evaluate_on_db(rows, app, batches=(8,), local=0, ensemble=3, seed=0):
    """Replay ``learned_tune`` on recorded measurements of ``app``: the
    ranker only learns the times of the configurations it picks.  Returns
    (best picked ms / best recorded ms, number measured, distinct plans)."""
    uniq = {}
    for r in rows:
        if r['app'] != app:
            continue
        k = signature(r['features'], r)
        if k not in uniq or r['ms'] < uniq[k]['ms']:
            uniq[k] = r
    te = list(uniq.values())
    Xc = app_normalized(np.stack([featurize(r['features'], r,
                                            pixels_of(r['data']))
                                  for r in te]), [0] * len(te))
    Xb, yb = db_training_set(rows, exclude_app=app)
    ranker = OnlineRanker(Xc, Xb, yb, ensemble=ensemble, seed=seed)
    best = ranker.run(te, lambda idx: [te[i]['ms'] for i in idx],
                      batches=batches, local=local)
    top = min(r['ms'] for r in te)
    return ranker.measured[best] / top, len(ranker.measured), len(te)
