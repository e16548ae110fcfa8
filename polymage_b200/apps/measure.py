"""Throughput of the shipped pipelines at their benchmark sizes on the GPU.

  python -m polymage_b200.apps.measure --app harris --steps 50 --warmup 5

For each pipeline: synthetic inputs of the benchmark size (seeded), the
default build from the catalog, device buffers, and ``--steps`` timed runs
of the whole pipeline (every group's launch) through ``pipeline_<name>_graph``
(the pipeline's kernels as one CUDA graph; ``graph=False``: ``_dev``).
Before each timed run a 256 MB buffer is written so that no input is still
in the 126 MB L2; each run is bracketed by CUDA events on the launching
stream.  Reported per pipeline: mean pipeline time, MPix/s (spatial pixels
of the output, rows x cols), and the compulsory-bytes roofline: (input
bytes + output bytes) / time against the measured HBM copy bandwidth.
"""

import argparse
import json
import os

import numpy as np

from . import catalog

APPS = ("harris", "unsharp", "campipe", "bilateral", "pyramid", "pyramid8",
        "laplacian")
# the pipelines beyond the benchmark configurations, at the reference
# Makefiles' sizes (catalog); for the grids "pixels" are the interior
# points a call updates
WIDENING = ("interpolate", "jacobi2d", "jacobi3d", "vcycle", "wcycle",
            "vcycle3d", "wcycle3d", "mg3p", "nlmeans", "maxfilter")
FLUSH_BYTES = 256 << 20


def workload(app, seed=0, size=None):
    """(params, host inputs, output shapes/dtypes, pixels, description).
    ``size``: (rows, cols) instead of the benchmark size (max filter only,
    for small profiling runs)."""
    rng = np.random.default_rng(seed)
    if size is not None and app != 'maxfilter':
        raise ValueError("a size can be given for the max filter only")
    if app == 'harris':
        n = 2048
        return ({'R': n - 2, 'C': n - 2},
                {'img': rng.random((n, n), dtype=np.float32)},
                {'harris': ((n, n), np.float32)}, n * n,
                "harris 2048x2048 float32")
    if app == 'unsharp':
        n = 4096
        img = np.zeros((3, n + 4, n + 4), np.float32)
        img[:, 2:n + 2, 2:n + 2] = rng.random((3, n, n), dtype=np.float32)
        return ({'R': n, 'C': n, 'threshold': 0.001, 'weight': 3.0},
                {'img': img}, {'mask': ((3, n, n), np.float32)}, n * n,
                "unsharp_mask 3x4096x4096 float32")
    if app == 'campipe':
        R, C = 1968, 2592
        from .campipe import MATRIX_3200, MATRIX_7000
        return ({'R': R, 'C': C, 'colour_temp': 3700.0, 'contrast': 50.0,
                 'gamma': 2.0},
                {'img': rng.integers(0, 1024, (R, C), dtype=np.int16),
                 'matrix_3200': np.asarray(MATRIX_3200, np.float32),
                 'matrix_7000': np.asarray(MATRIX_7000, np.float32)},
                {'process': ((3, R - 48, C - 64), np.uint8)},
                (R - 48) * (C - 64),
                "camera_pipe 2592x1968 uint16 raw -> uint8 RGB")
    if app == 'bilateral':
        rows, cols = 1536, 2560
        return ({'rows': rows, 'cols': cols},
                {'input': rng.random((rows, cols), dtype=np.float32)},
                {'filtered': ((1, rows, cols), np.float32)}, rows * cols,
                "bilateral_grid 2560x1536 float32")
    if app == 'pyramid':
        R = C = 2108
        return ({'R': R, 'C': C},
                {'img1': rng.random((3, R, C), dtype=np.float32),
                 'img2': rng.random((3, R, C), dtype=np.float32),
                 'mask': rng.random((R, C), dtype=np.float32)},
                {'blend': ((3, R - 60, C - 60), np.float32)},
                (R - 60) * (C - 60),
                "pyramid_blend L=4 3x2108x2108 float32")
    if app == 'pyramid8':
        R = C = 2048
        return ({'R': R, 'C': C},
                {'img1': rng.random((3, R, C), dtype=np.float32),
                 'img2': rng.random((3, R, C), dtype=np.float32),
                 'mask': rng.random((R, C), dtype=np.float32)},
                {'blend': ((3, R, C), np.float32)}, R * C,
                "pyramid_blend L=8 (clamped borders) 3x2048x2048 float32")
    if app == 'laplacian':
        H, W = 1080, 1920
        return ({'R': H + 92, 'C': W + 92, 'alpha': 1.0 / 3.0, 'beta': 1.0},
                {'img_colour': rng.integers(0, 256, (H, W, 3),
                                            dtype=np.uint8)},
                {'laplacian': ((H, W, 3), np.uint8)}, H * W,
                "local_laplacian 1920x1080 uint8 BGR, 4 intensity levels, "
                "5 pyramid levels")
    if app == 'interpolate':
        R = C = 2048
        img = np.zeros((4, R + 2, C + 2), np.float32)
        img[0:3, 1:R + 1, 1:C + 1] = rng.random((3, R, C), dtype=np.float32)
        img[3, 1:R + 1, 1:C + 1] = 0.25 + 0.75 * rng.random(
            (R, C), dtype=np.float32)
        return ({'R': R, 'C': C}, {'img': img},
                {'interpolate': ((3, R, C), np.float32)}, R * C,
                "interpolate 2048x2048 RGBA float32, 10 levels")
    if app in ('jacobi2d', 'jacobi3d'):
        kw = catalog.JACOBI2D if app == 'jacobi2d' else catalog.JACOBI3D
        N, dims = kw['N'], 2 if app == 'jacobi2d' else 3
        shape = (N + 2,) * dims
        return ({'N': N}, {'V_': rng.random(shape), 'F_': rng.random(shape)},
                {'jacobi': (shape, np.float64)}, N ** dims,
                "jacobi %dD N=%d float64, %d steps" % (dims, N, kw['T']))
    if app in ('vcycle', 'wcycle', 'vcycle3d', 'wcycle3d'):
        kw = catalog._BUILDERS[app][1]
        n, L, dims = kw['n'], kw['L'], kw.get('dims', 2)
        N = (n + 1) * (1 << L) - 1
        shape = (N + 2,) * dims
        out = {'vcycle': 'Vcycle', 'wcycle': 'Wcycle',
               'vcycle3d': 'Vcycle3d', 'wcycle3d': 'Wcycle3d'}[app]
        return ({'n': n}, {'V_': rng.random(shape), 'F_': rng.random(shape)},
                {out: (shape, np.float64)}, N ** dims,
                "%s-cycle %dD finest %d^%d float64, L=%d nu1=%d nu2=%d "
                "nuc=%d" % ('W' if kw.get('gamma', 1) == 2 else 'V', dims, N,
                            dims, L, kw['nu1'], kw['nu2'], kw['nuc']))
    if app == 'mg3p':
        from .nas_mg import SIZES
        n = SIZES[catalog.MG3P['prob_class']]
        shape = (n + 2,) * 3
        return ({'n': n}, {'U': rng.random(shape), 'V': rng.random(shape),
                           'R': rng.random(shape)},
                {'MG_U': (shape, np.float64), 'MG_R': (shape, np.float64)},
                n ** 3, "NAS MG mg3P class %s (%d^3) float64"
                % (catalog.MG3P['prob_class'], n))
    if app == 'maxfilter':
        R, C = size or (catalog.MAXFILTER['rows'], catalog.MAXFILTER['cols'])
        return ({'R': R, 'C': C},
                {'img': rng.integers(0, 256, (3, R, C)).astype(np.float32)},
                {'final': ((R, C, 3), np.int32)}, R * C,
                "max_filter %dx%d RGB (0..255 as float32), radius 26" % (
                    R, C))
    if app == 'nlmeans':
        R, C = catalog.NLMEANS['rows'], catalog.NLMEANS['cols']
        x = np.arange(R)[:, None] / R
        y = np.arange(C)[None, :] / C
        img = np.empty((3, R, C), np.float32)
        for c in range(3):
            img[c] = 0.5 + 0.3 * np.sin(6.0 * x + 2.0 * c) * \
                np.cos(5.0 * y) + 0.02 * rng.standard_normal((R, C))
        return ({'R': R, 'C': C, 'patch_size': 7, 'search_area': 7},
                {'img': img}, {'non_local_means': ((3, R, C), np.float32)},
                R * C, "non_local_means %dx%d RGB float32, patch 7, search "
                "area 7" % (R, C))
    raise ValueError(app)


def hbm_peak():
    root = os.path.dirname(os.path.dirname(os.path.dirname(
        os.path.abspath(__file__))))
    p = os.path.join(root, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measure(app, steps=50, warmup=5, device=None, graph=True, warm=False,
            cp=None, size=None):
    """Mean device time of ``steps`` runs of one shipped pipeline at its
    benchmark size (CUDA events on the launching stream).  By default 256 MB
    are written before each run so that nothing starts in L2; ``warm``
    leaves the previous run's data in L2 (the sub-L2 workloads' warm
    numbers).  ``cp``: another build of the same pipeline (a variant of
    the catalog's) to time instead of the catalog's."""
    import torch
    dev = device or torch.device("cuda", torch.cuda.current_device())
    cp = cp or catalog.build(app)
    prm, host_in, out_spec, pixels, desc = workload(app, size=size)
    # inputs that only const tables read (the camera pipe's two 3x4 colour
    # matrices) stay in host memory, where the tables are computed
    table_only = set(f.name for f in cp.inputs if id(f) in cp.table_only)
    ins = dict((k, torch.from_numpy(v) if k in table_only
                else torch.from_numpy(v).to(dev))
               for k, v in host_in.items())
    outs = {}
    for k, (shape, dt) in out_spec.items():
        outs[k] = torch.zeros(shape, dtype=torch.from_numpy(
            np.zeros(1, dt)).dtype, device=dev)
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    if graph:
        from ..runtime import PipelineRuntimeError
        try:
            cp.run_dev(prm, ins, outs, stream=stream.cuda_stream, graph=True)
        except PipelineRuntimeError:
            # no graph form (const tables computed from input contents)
            graph = False
    for _ in range(max(warmup, 3)):
        cp.run_dev(prm, ins, outs, stream=stream.cuda_stream, graph=graph)
    torch.cuda.synchronize(dev)
    cp.check()
    ev = [(torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for i in range(steps):
        if not warm:
            flush.fill_(float(i))
        ev[i][0].record(stream)
        cp.run_dev(prm, ins, outs, stream=stream.cuda_stream, graph=graph)
        ev[i][1].record(stream)
    torch.cuda.synchronize(dev)
    cp.check()
    per = sorted(a.elapsed_time(b) for a, b in ev)
    ms = float(np.mean(per))
    nbytes = sum(v.nbytes for v in host_in.values()) + sum(
        int(np.prod(s)) * np.dtype(d).itemsize for s, d in out_spec.values())
    peak, kind = hbm_peak()
    gbs = nbytes / (ms / 1e3) / 1e9
    return {"app": app, "workload": desc, "ms": ms,
            "ms_min": per[0], "ms_median": float(np.median(per)),
            "ms_max": per[-1],
            "mpix_s": pixels / (ms / 1e3) / 1e6,
            "launches": cp.module.meta.get('launches'),
            "entry": "pipeline_%s_%s" % (cp.name, "graph" if graph else "dev"),
            "compulsory_bytes": int(nbytes), "achieved_gbs": gbs,
            "hbm_frac": gbs / peak, "peak_gbs": peak, "peak_source": kind,
            "l2": ("warm: the previous run's data left in L2" if warm else
                   "256 MB written before each timed run")}


def int_peak(device=None, iters=4096, steps=20):
    """Integer-ALU throughput of the GPU (thread instructions per second)
    from polymage_b200/csrc/int_peak.cu: 8 independent 32-bit
    multiply-add chains (IMAD) or add/xor chains per thread, 148 x 16
    CTAs of 256 threads, CUDA events, best of ``steps`` runs.  Each round
    of the IMAD kernel is 8 integer instructions per thread and of the ALU
    kernel 18 (8 adds, 8 xors, and the two updates of its operands)."""
    import ctypes
    import torch
    from ..build import compile_source
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lib = ctypes.CDLL(compile_source("int_peak", os.path.join(
        here, "csrc", "int_peak.cu")))
    lib.pm_int_peak_run.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p,
                                                         ctypes.c_void_p]
    dev = device or torch.device("cuda", torch.cuda.current_device())
    blocks = 148 * 16
    out = torch.empty(blocks * 256, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    res = {}
    for which, name, per_round in ((0, "imad", 8), (1, "add_xor", 18)):
        best = None
        for i in range(steps + 2):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            if lib.pm_int_peak_run(which, blocks, iters, out.data_ptr(),
                                   stream.cuda_stream) != 0:
                raise RuntimeError("int_peak launch failed")
            b.record(stream)
            torch.cuda.synchronize(dev)
            if i >= 2:
                ms = a.elapsed_time(b)
                best = ms if best is None else min(best, ms)
        n = float(blocks) * 256 * iters * per_round
        res[name] = {"ms": best, "thread_inst_per_s": n / (best / 1e3),
                     "thread_inst_per_launch": n}
    return res


def measure_host(app, steps=10, warmup=2):
    """End to end through the reference's C ABI (``pipeline_<name>`` on
    pinned host buffers: copies to and from the device inside the call),
    host wall clock over ``steps`` calls, as bench.py's ``e2e``."""
    import time
    import torch
    cp = catalog.build(app)
    prm, host_in, out_spec, pixels, desc = workload(app)
    ins = {}
    for k, v in host_in.items():
        t = torch.from_numpy(v).pin_memory()
        ins[k] = t.numpy()
    outs = {}
    for k, (shape, dt) in out_spec.items():
        t = torch.zeros(shape, dtype=torch.from_numpy(
            np.zeros(1, dt)).dtype).pin_memory()
        outs[k] = t.numpy()
    for _ in range(warmup):
        cp.run_host(prm, ins, outs)
    s0 = time.perf_counter()
    for _ in range(steps):
        cp.run_host(prm, ins, outs)
    sec = (time.perf_counter() - s0) / steps
    h2d = sum(v.nbytes for v in ins.values())
    d2h = sum(v.nbytes for v in outs.values())
    return {"app": app, "workload": desc, "api": "pipeline_%s (host "
            "buffers, pinned)" % cp.name, "ms": sec * 1e3,
            "mpix_s": pixels / sec / 1e6, "h2d_bytes": int(h2d),
            "d2h_bytes": int(d2h)}


def measure_bilateral_batch(n=64, steps=10, warmup=3, graph=True,
                            device=None, seed=1):
    """The batched bilateral-grid workload: ``n`` images whose sides are
    drawn uniformly from 512..4096 (seeded), each U[0,1), run as one batch
    (one launch per group, persistent tile queue) through
    ``pipeline_bilateral_batch_graph`` (or ``_batch``).  Inputs are created
    on the device; timed with CUDA events, L2 flushed before each run."""
    import torch
    dev = device or torch.device("cuda", torch.cuda.current_device())
    cp = catalog.build("bilateral")
    rng = np.random.default_rng(seed)
    sides = rng.integers(512, 4097, (n, 2))
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    prms, ins, outs = [], [], []
    for r, c in sides:
        r, c = int(r), int(c)
        prms.append({'rows': r, 'cols': c})
        ins.append({'input': torch.rand((r, c), generator=gen, device=dev)})
        outs.append({'filtered': torch.zeros((1, r, c), device=dev)})
    pixels = float(sum(int(r) * int(c) for r, c in sides))
    nbytes = pixels * 8
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(max(warmup, 3)):
        cp.run_batch(prms, ins, outs, stream=stream.cuda_stream, graph=graph)
    torch.cuda.synchronize(dev)
    cp.check()
    ev = [(torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for i in range(steps):
        flush.fill_(float(i))
        ev[i][0].record(stream)
        cp.run_batch(prms, ins, outs, stream=stream.cuda_stream, graph=graph)
        ev[i][1].record(stream)
    torch.cuda.synchronize(dev)
    cp.check()
    ms = float(np.mean([a.elapsed_time(b) for a, b in ev]))
    peak, kind = hbm_peak()
    gbs = nbytes / (ms / 1e3) / 1e9
    return {"app": "bilateral_batch%d" % n,
            "workload": "bilateral_grid batch of %d images, sides "
                        "U{512..4096} seed %d, %.1f MPix" % (n, seed,
                                                             pixels / 1e6),
            "ms": ms, "mpix_s": pixels / (ms / 1e3) / 1e6,
            "entry": "pipeline_bilateral_batch_graph" if graph
            else "pipeline_bilateral_batch",
            "compulsory_bytes": int(nbytes), "achieved_gbs": gbs,
            "hbm_frac": gbs / peak, "peak_gbs": peak, "peak_source": kind,
            "l2": "256 MB written before each timed run"}


def measure_stream(n=1024, seed=1, device=None):
    """The mixed request stream (``polymage_b200.apps.stream``): ``n``
    Harris / unsharp / pyramid requests with sides U{256..4096}, served in
    per-pipeline batches; MPix/s and compulsory-bytes roofline over the
    batch calls' GPU time (second of two passes over the stream)."""
    from . import stream
    reqs = stream.make_stream(n, seed)
    # a first pass sizes the batch workspaces and descriptor buffers (their
    # allocations would otherwise fall inside the timed batch calls)
    stream.serve(reqs, device=device, seed=seed)
    r = stream.serve(reqs, device=device, seed=seed)
    peak, kind = hbm_peak()
    gbs = r["bytes"] / (r["ms"] / 1e3) / 1e9
    return {"app": "stream%d" % n,
            "workload": "%d requests (Harris, unsharp, pyramid L=8), sides "
                        "U{256..4096} seed %d, %.1f GPix" % (
                            n, seed, r["pixels"] / 1e9),
            "ms": r["ms"], "mpix_s": r["pixels"] / (r["ms"] / 1e3) / 1e6,
            "chunks": r["chunks"], "batch_calls": r["batch_calls"],
            "compulsory_bytes": int(r["bytes"]), "achieved_gbs": gbs,
            "hbm_frac": gbs / peak, "peak_gbs": peak, "peak_source": kind,
            "l2": "inputs of each chunk (8 GB) larger than L2"}


def parse_options(text):
    """Build options from a JSON list: lists become the tuples options are
    written with, at every depth (``[["storage_order", [["vert", [3, 0, 1,
    2]]]]]`` is ``[('storage_order', (('vert', (3, 0, 1, 2)),))]``)."""
    def tup(o):
        return tuple(tup(x) for x in o) if isinstance(o, list) else o
    return [tup(o) for o in json.loads(text or "[]")]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--app", action="append",
                    choices=APPS + WIDENING + ("bilateral_batch64",
                                               "stream1024"))
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--warm", action="store_true",
                    help="no L2 flush between runs (single-image pipelines)")
    ap.add_argument("--host", action="store_true",
                    help="end to end through the host-buffer C ABI")
    ap.add_argument("--int-peak", action="store_true",
                    help="integer-ALU throughput of the GPU")
    ap.add_argument("--options", default=None,
                    help="JSON list of options added to the catalog build "
                         "(e.g. '[\"chain\"]')")
    ap.add_argument("--drop-options", default=None,
                    help="JSON list of catalog options left out")
    ap.add_argument("--size", type=int, nargs=2, default=None,
                    metavar=("ROWS", "COLS"),
                    help="another image size (max filter only)")
    args = ap.parse_args()
    if args.int_peak:
        print(json.dumps(int_peak()))
        return
    for app in args.app or APPS + ("bilateral_batch64", "stream1024"):
        if app == "stream1024":
            print(json.dumps(measure_stream(1024)))
        elif app == "bilateral_batch64":
            print(json.dumps(measure_bilateral_batch(
                64, steps=min(args.steps, 10), warmup=args.warmup)))
        elif args.host:
            print(json.dumps(measure_host(app, min(args.steps, 20))))
        else:
            cp = None
            add = parse_options(args.options)
            drop = parse_options(args.drop_options)
            if add or drop:
                cp = catalog.variant(app, add, drop).build()
            r = measure(app, args.steps, args.warmup, warm=args.warm, cp=cp,
                        size=tuple(args.size) if args.size else None)
            if add or drop:
                r["options"] = add
                r["dropped"] = drop
            print(json.dumps(r))


if __name__ == "__main__":
    main()
