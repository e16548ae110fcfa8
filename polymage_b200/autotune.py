"""Tune the shipped pipelines on synthetic inputs of their benchmark sizes.

  python -m polymage_b200.autotune --app unsharp --db timing_db.jsonl
  python -m polymage_b200.autotune --app harris --learned model.npz --k 5

Exhaustive mode runs ``tuner.generate`` + ``tuner.execute`` over the
reference's search space (15 tile shapes x the 5 group sizes the
reference's app tuners use, harris/app_tuner.py:33-54, plus 11, the size
that fuses Harris whole) times the register blocking options, appending
every measurement to the timing database.
Learned mode ranks the same space with the cost model (pretrained on the
other pipelines' measurements) and compiles and times only its top picks
(8 by default), in one round.
"""

import argparse
import json
import os
import time

import numpy as np

from . import tuner
from .apps.harris import harris_pipe
from .apps.unsharp_mask import unsharp_mask
from .apps.campipe import camera_pipe, MATRIX_3200, MATRIX_7000
from .apps.bilateral_grid import bilateral_grid
from .apps.pyramid_blend import pyramid_blending, pyramid_blending_clamped
from .constructs import Condition


def app_setup(app, seed=0):
    """(tuner arg dict, pipe arg data) for one shipped pipeline."""
    rng = np.random.default_rng(seed)
    d = {}
    if app == 'harris':
        out = harris_pipe(d)
        rows = cols = 2048
        est = [(d['R'], rows - 2), (d['C'], cols - 2)]
        data = {'R': rows - 2, 'C': cols - 2,
                'img': rng.random((rows, cols), dtype=np.float32),
                'harris': np.zeros((rows, cols), np.float32)}
    elif app == 'unsharp':
        out = unsharp_mask(d)
        R = C = 4096
        est = [(d['R'], R), (d['C'], C)]
        data = {'R': R, 'C': C, 'threshold': 0.001, 'weight': 3.0,
                'img': rng.random((3, R + 4, C + 4), dtype=np.float32),
                'mask': np.zeros((3, R, C), np.float32)}
    elif app == 'campipe':
        out = camera_pipe(d)
        R, C = 1968, 2592
        est = [(d['R'], R), (d['C'], C)]
        m3 = np.array(MATRIX_3200, np.float32)
        m7 = np.array(MATRIX_7000, np.float32)
        data = {'C': C, 'R': R, 'colour_temp': 3700.0, 'contrast': 50.0,
                'gamma': 2.0,
                'img': rng.integers(0, 1024, (R, C), dtype=np.int16),
                'matrix_3200': m3, 'matrix_7000': m7,
                'process': np.zeros((3, R - 48, C - 64), np.uint8)}
    elif app == 'bilateral':
        out = bilateral_grid(d)
        rows, cols = 1536, 2560
        est = [(d['R'], rows), (d['C'], cols)]
        data = {'rows': rows, 'cols': cols,
                'input': rng.random((rows, cols), dtype=np.float32),
                'filtered': np.zeros((1, rows, cols), np.float32)}
    elif app == 'pyramid':
        out = pyramid_blending(d)
        R = C = 2108
        est = [(d['R'], R), (d['C'], C)]
        data = {'R': R, 'C': C,
                'img1': rng.random((3, R, C), dtype=np.float32),
                'img2': rng.random((3, R, C), dtype=np.float32),
                'mask': rng.random((R, C), dtype=np.float32),
                'blend': np.zeros((3, R - 60, C - 60), np.float32)}
    elif app == 'pyramid8':
        out = pyramid_blending_clamped(d, L=8)
        R = C = 2048
        est = [(d['R'], R), (d['C'], C)]
        data = {'R': R, 'C': C,
                'img1': rng.random((3, R, C), dtype=np.float32),
                'img2': rng.random((3, R, C), dtype=np.float32),
                'mask': rng.random((R, C), dtype=np.float32),
                'blend': np.zeros((3, R, C), np.float32)}
    else:
        raise ValueError(app)
    arg = {'_tuner_app_name': app, '_tuner_live_outs': [out],
           '_tuner_param_estimates': est,
           '_tuner_param_constraints': [Condition(p, '==', v)
                                        for p, v in est],
           '_tuner_tile_size_configs': tuner.DEFAULT_TILES,
           '_tuner_group_size_configs': tuner.DEFAULT_GROUPS,
           '_tuner_option_configs': [['rblock=4']],
           '_tuner_pipe_arg_data': data,
           '_tuner_debug_flag': False}
    if app == 'bilateral':
        arg['_tuner_opts'] = [('red_tile', (32, 256))]
    return arg


def exhaustive(app, db, dst, nruns=5, option_configs=None):
    a = app_setup(app)
    if option_configs is not None:
        a['_tuner_option_configs'] = option_configs
    a['_tuner_dst_path'] = dst
    a['_tuner_db'] = db
    t0 = time.time()
    src, n, pipe = tuner.generate(a)
    t1 = time.time()
    a['_tuner_src_path'] = src
    a['_tuner_pipe'] = pipe
    a['_tuner_nruns'] = nruns
    rep = tuner.execute(a)
    t2 = time.time()
    rep['generate_s'] = t1 - t0
    rep['wall_s'] = t2 - t0
    return rep


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--app', required=True)
    ap.add_argument('--db', default='timing_db.jsonl')
    ap.add_argument('--dst', default='/tmp')
    ap.add_argument('--nruns', type=int, default=5)
    ap.add_argument('--learned', action='store_true',
                    help='online learned tuning (cost model)')
    ap.add_argument('--compare', action='store_true',
                    help='learned tuning, then exhaustive tuning to compare')
    ap.add_argument('--picks', type=int, default=8,
                    help='configurations the learned tuner times (one '
                         'compile round)')
    ap.add_argument('--options', default=None,
                    help='JSON list of option lists to search over')
    ap.add_argument('--report', default=None)
    ap.add_argument('--train-db', default=None,
                    help='timing database the learned tuner pretrains on '
                         '(other pipelines\' rows; default: the shipped one)')
    args = ap.parse_args()
    opts = json.loads(args.options) if args.options else None
    out = {'app': args.app}
    if args.learned or args.compare:
        from .costmodel import learned_tune
        a = app_setup(args.app)
        if opts is not None:
            a['_tuner_option_configs'] = opts
        a['_tuner_dst_path'] = os.path.join(args.dst, 'learned')
        a['_tuner_nruns'] = args.nruns
        rows = tuner.load_db(args.train_db) if args.train_db else None
        lr = learned_tune(a, db_rows=rows, batches=(args.picks,), local=0,
                          shipped_app=args.app)
        out['learned'] = {'best': lr['best'], 'best_ms': lr['best_ms'],
                          'wall_s': lr['wall_s'], 'plan_s': lr['plan_s'],
                          'compile_s': lr['compile_s'],
                          'time_s': lr['time_s'],
                          'measured': len(lr['measured']),
                          'candidates': lr['candidates']}
    if not args.learned or args.compare:
        rep = exhaustive(args.app, args.db, args.dst, args.nruns,
                         option_configs=opts)
        best = rep['results'][0] if rep['results'] else None
        out['exhaustive'] = {'best': best, 'wall_s': rep['wall_s'],
                             'generate_s': rep['generate_s'],
                             'n': len(rep['results'])}
    if args.compare and out['exhaustive']['best'] and \
            out['learned']['best_ms']:
        out['time_ratio'] = out['learned']['best_ms'] / \
            out['exhaustive']['best']['ms']
        out['wall_ratio'] = out['learned']['wall_s'] / \
            out['exhaustive']['wall_s']
    if args.report:
        with open(args.report, 'w') as f:
            json.dump(out, f, indent=1)
    print(json.dumps(out))


if __name__ == '__main__':
    main()
