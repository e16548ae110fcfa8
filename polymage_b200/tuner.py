"""Autotuner: exhaustive search over tile sizes x group sizes (x extra
CUDA-target options), with the reference's interface
(sandbox/tuner.py:100-631):

* ``generate(arg_data)`` builds a pipeline per configuration and compiles
  it (here: nvcc for sm_100a, several builds in parallel); a configuration
  whose plan or build fails is logged and skipped (:302-319, :343-353).
  Returns ``(src_path, configs_count, pipe)``.
* ``execute(arg_data)`` runs every compiled configuration ``nruns`` times on
  the same inputs and keeps the minimum time (:510-598); it reports the
  global best (:615-626) and writes a report.  Timing is by CUDA events on
  device-resident buffers instead of ``time.time()`` around a host call.

Keys are the reference's ``_tuner_*`` keys; ``_tuner_omp_threads`` and
``_tuner_cxx_string`` are accepted and ignored.  Additions:
``_tuner_option_configs`` (lists of extra options, e.g. register blocking),
``_tuner_jobs`` (parallel builds), ``_tuner_db`` (JSONL timing database:
every measured configuration is appended with its plan features, so tuning
resumes and the learned cost model trains on it).
"""

import hashlib
import itertools
import json
import os
import sys
import time
from concurrent.futures import ThreadPoolExecutor

from .compiler import buildPipeline
from .tiling import PlanError

DEFAULT_TILES = [[64, 256], [64, 128], [32, 512], [32, 256], [32, 128],
                 [32, 64], [16, 512], [16, 256], [16, 128], [16, 64],
                 [8, 512], [8, 256], [8, 128], [8, 64], [8, 32]]
DEFAULT_GROUPS = [3, 5, 7, 9, 10, 11]


def _log(dump, msg):
    for f in dump:
        print(msg, file=f)
        f.flush()


def config_key(app, cfg):
    s = json.dumps([app, cfg['tile'], cfg['group_size'],
                    [list(o) if isinstance(o, tuple) else o
                     for o in cfg['options']]], sort_keys=True)
    return hashlib.sha1(s.encode()).hexdigest()[:16]


def enumerate_configs(tiles, groups, option_configs):
    out = []
    for t, g, o in itertools.product(tiles, groups, option_configs or [[]]):
        out.append({'tile': list(t), 'group_size': int(g),
                    'options': list(o)})
    return out


def plan_config(a, cfg, name):
    """Build (plan only, no compile) the pipeline of one configuration."""
    return buildPipeline(a['_tuner_live_outs'],
                         param_estimates=a.get('_tuner_param_estimates')
                         or [],
                         param_constraints=a.get('_tuner_param_constraints')
                         or [],
                         tile_sizes=cfg['tile'],
                         group_size=cfg['group_size'],
                         options=list(a.get('_tuner_opts') or []) +
                         list(cfg['options']),
                         pipe_name=name)


def generate(_tuner_arg_data):
    from .build import compile_module, BuildError
    a = _tuner_arg_data
    app = a['_tuner_app_name']
    name = a.get('_tuner_pipe_name') or app
    tiles = a.get('_tuner_tile_size_configs') or DEFAULT_TILES
    groups = a.get('_tuner_group_size_configs') or DEFAULT_GROUPS
    dst = a.get('_tuner_dst_path') or '/tmp'
    jobs = int(a.get('_tuner_jobs') or max(1, (os.cpu_count() or 2) // 2))
    dump = [sys.stdout] if a.get('_tuner_debug_flag') else []
    configs = a.get('_tuner_configs') or enumerate_configs(
        tiles, groups, a.get('_tuner_option_configs'))
    src_path = os.path.join(dst, "PolyB200Tune_%s" % app)
    os.makedirs(src_path, exist_ok=True)
    t0 = time.time()
    manifest = []
    modules = []
    first_pipe = None
    for i, cfg in enumerate(configs):
        entry = dict(cfg, id=i, key=config_key(app, cfg), so=None,
                     status='planned')
        try:
            p = plan_config(a, cfg, name)
            entry['features'] = pipeline_features(p)
            entry['ngroups'] = len(p.groups)
            mod = p.generate_code()
            modules.append((entry, mod))
            if first_pipe is None:
                first_pipe = p
        except (PlanError, TypeError, ValueError) as e:
            entry['status'] = 'plan_failed'
            entry['error'] = str(e)[:200]
            _log(dump, "tuner: config %d %s %s: plan failed (%s)" % (
                i, cfg['tile'], cfg['group_size'], e))
        manifest.append(entry)

    def build(item):
        entry, mod = item
        try:
            entry['so'] = compile_module(mod)
            entry['status'] = 'built'
        except Exception as e:          # a failing build is skipped
            entry['status'] = 'build_failed'
            entry['error'] = str(e)[-300:]
        return entry

    with ThreadPoolExecutor(max_workers=jobs) as ex:
        for entry in ex.map(build, modules):
            _log(dump, "tuner: config %d tile %s group %d: %s" % (
                entry['id'], entry['tile'], entry['group_size'],
                entry['status']))
    elapsed = time.time() - t0
    with open(os.path.join(src_path, "configurations.json"), "w") as f:
        json.dump({'app': app, 'name': name, 'generate_s': elapsed,
                   'configs': manifest}, f, indent=1)
    with open(os.path.join(src_path, "configurations.txt"), "w") as f:
        for e in manifest:
            f.write("%d %s group_size=%d options=%s %s\n" % (
                e['id'], e['tile'], e['group_size'], e['options'],
                e['status']))
    built = sum(1 for e in manifest if e['status'] == 'built')
    _log(dump, "tuner: generated %d configurations (%d built) in %.1f s" % (
        len(manifest), built, elapsed))
    return src_path, len(manifest), first_pipe


def pipeline_features(pipe):
    """Numeric description of a built pipeline (sum/max over its fused
    groups) for the cost model."""
    feats = {'ngroups': 0, 'nstencil': 0, 'nred': 0, 'stages': 0,
             'smem_max': 0, 'smem_sum': 0, 'halo_max': 0.0,
             'redund_sum': 0.0, 'tile_inner': 0, 'tile_outer': 0,
             'threads': 0, 'cost_sum': 0, 'nsmem': 0, 'nstage_in': 0,
             'ninline': 0}
    for g in pipe.groups:
        feats['ngroups'] += 1
        f = g.plan.features() if g.plan is not None else {}
        if g.kind == 'stencil':
            feats['nstencil'] += 1
        elif g.kind == 'reduction':
            feats['nred'] += 1
        feats['stages'] += f.get('nstages', 0)
        feats['smem_max'] = max(feats['smem_max'], f.get('smem_bytes', 0))
        feats['smem_sum'] += f.get('smem_bytes', 0)
        feats['halo_max'] = max(feats['halo_max'], f.get('halo', 0.0))
        feats['redund_sum'] += f.get('redundancy', 0.0)
        feats['tile_inner'] = max(feats['tile_inner'], f.get('tile_inner',
                                                              0))
        feats['tile_outer'] = max(feats['tile_outer'], f.get('tile_outer',
                                                              0))
        feats['threads'] = max(feats['threads'], f.get('threads', 0))
        feats['cost_sum'] += f.get('cost', 0)
        feats['nsmem'] += f.get('nsmem', 0)
        feats['nstage_in'] += f.get('nstage_in', 0)
        feats['ninline'] += f.get('ninline', 0)
    return feats


# ---------------------------------------------------------------------------
_flush_buf = None


def _flush_l2(stream):
    """Write a 256 MB buffer (twice the 126 MB L2) so that a timed run
    starts with none of its inputs or intermediates cached."""
    global _flush_buf
    import torch
    if _flush_buf is None:
        _flush_buf = torch.empty(64 << 20, dtype=torch.float32,
                                 device=torch.cuda.current_device())
    with torch.cuda.stream(stream):
        _flush_buf.fill_(0.0)


def _time_config(so_path, pipe_name, params, dev_inputs, dev_outputs, nruns,
                 warmup=2):
    """min-of-nruns device time (ms) of one compiled configuration, L2
    flushed before every timed run."""
    import ctypes
    import torch
    from . import constructs as C
    lib = ctypes.CDLL(so_path)
    fn = getattr(lib, "pipeline_%s_dev" % pipe_name)
    fn.restype = ctypes.c_int
    ordered = params['_ordered']
    args = []
    types = []
    for p in ordered[0]:
        if p.typ in (C.Float, C.Double):
            args.append(float(params[p.name]))
            types.append(ctypes.c_float)
        else:
            args.append(int(params[p.name]))
            types.append(ctypes.c_int)
    for f in ordered[1]:
        args.append(dev_inputs[f.name].data_ptr())
        types.append(ctypes.c_void_p)
    for f in ordered[2]:
        args.append(dev_outputs[f.name].data_ptr())
        types.append(ctypes.c_void_p)
    stream = torch.cuda.current_stream()
    args.append(stream.cuda_stream)
    types.append(ctypes.c_void_p)
    fn.argtypes = types
    for _ in range(warmup):
        st = fn(*args)
        if st != 0:
            raise RuntimeError("status %d" % st)
    torch.cuda.synchronize()
    best = None
    for _ in range(nruns):
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        _flush_l2(stream)
        s.record(stream)
        fn(*args)
        e.record(stream)
        torch.cuda.synchronize()
        ms = s.elapsed_time(e)
        best = ms if best is None else min(best, ms)
    return best


def execute(_tuner_arg_data):
    """Time every built configuration of a ``generate`` run; returns the
    report dict (best configuration first)."""
    import torch
    a = _tuner_arg_data
    app = a['_tuner_app_name']
    src = a.get('_tuner_src_path') or '/tmp'
    nruns = int(a.get('_tuner_nruns') or 1)
    dump = [sys.stdout] if a.get('_tuner_debug_flag', True) else []
    only = a.get('_tuner_only_ids')
    with open(os.path.join(src, "configurations.json")) as f:
        man = json.load(f)
    pipe = a['_tuner_pipe']
    data = a['_tuner_pipe_arg_data']
    custom = a.get('_tuner_custom_executor')
    params = dict((k, v) for k, v in data.items()
                  if not hasattr(v, 'shape'))
    params['_ordered'] = pipe.ordered_params()
    dev = torch.device('cuda', torch.cuda.current_device())
    dev_in = dict((f.name, _to_dev(data[f.name], dev))
                  for f in params['_ordered'][1])
    dev_out = dict((f.name, _to_dev(data[f.name], dev))
                   for f in params['_ordered'][2])
    db = a.get('_tuner_db')
    t0 = time.time()
    results = []
    for e in man['configs']:
        if e['status'] != 'built':
            continue
        if only is not None and e['id'] not in only:
            continue
        try:
            if custom is not None:
                ms = custom(e, a)
            else:
                ms = _time_config(e['so'], man['name'], params, dev_in,
                                  dev_out, nruns)
            e['ms'] = ms
            results.append(e)
            _log(dump, "tuner: config %d tile %s group %d %s: %.4f ms" % (
                e['id'], e['tile'], e['group_size'], e['options'], ms))
            if db:
                record(db, app, e, ms, data_key(data))
        except Exception as ex:      # a failing configuration is skipped
            _log(dump, "tuner: config %d failed to run: %s" % (e['id'], ex))
    elapsed = time.time() - t0
    results.sort(key=lambda r: r['ms'])
    report = {'app': app, 'execute_s': elapsed, 'nruns': nruns,
              'results': [dict((k, r[k]) for k in
                               ('id', 'tile', 'group_size', 'options', 'ms'))
                          for r in results]}
    stamp = time.strftime("%Y%m%d_%H%M%S")
    with open(os.path.join(src, "tuning_report_%s.json" % stamp), "w") as f:
        json.dump(report, f, indent=1)
    if results:
        b = results[0]
        _log(dump, "tuner: best config %d tile %s group %d %s: %.4f ms" % (
            b['id'], b['tile'], b['group_size'], b['options'], b['ms']))
    return report


def _to_dev(arr, dev):
    import torch
    return torch.from_numpy(arr).to(dev)


def data_key(data):
    shapes = sorted((k, list(v.shape)) for k, v in data.items()
                    if hasattr(v, 'shape'))
    return json.dumps(shapes)


def gpu_name():
    try:
        import torch
        return torch.cuda.get_device_name()
    except Exception:
        return "unknown"


def record(db_path, app, entry, ms, dkey):
    """Append one measurement to the JSONL timing database."""
    row = {'app': app, 'key': entry['key'], 'tile': entry['tile'],
           'group_size': entry['group_size'], 'options': entry['options'],
           'features': entry.get('features', {}), 'ms': ms, 'data': dkey,
           'gpu': gpu_name(), 'when': time.time()}
    os.makedirs(os.path.dirname(os.path.abspath(db_path)), exist_ok=True)
    with open(db_path, "a") as f:
        f.write(json.dumps(row) + "\n")


def load_db(db_path):
    rows = []
    if not os.path.exists(db_path):
        return rows
    with open(db_path) as f:
        for line in f:
            line = line.strip()
            if line:
                try:
                    rows.append(json.loads(line))
                except ValueError:
                    continue           # a torn last line is skipped
    return rows
