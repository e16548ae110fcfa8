"""Per-pipeline CPU baselines and reference outputs for the benchmark
workloads -- test infrastructure only: bench.py's cpu_baseline leg calls
it, as the checker and as the timed CPU baseline beside the GPU numbers.

For each shipped pipeline, on the inputs the GPU measurement uses
(``polymage_b200.apps.measure.workload``):

* ``expected(app, params, inputs)``: the oracle's outputs (FP64
  restatements; the camera pipe's C restatement, bit-exact; the local
  Laplacian's float32 restatement in the reference's operation order) and,
  where a select has a tie band, the mask of points outside it;
* ``time_baseline(app, params, inputs, threads)``: the CPU implementation
  timed on the host cores --
  - ``reference``: the reference's own generated C++ built from its tree
    (oracle/_ref): refHarris (sandbox/ipp_bench/harris/harris_function.cpp:
    9), pipeline_mask (sandbox/video_demo/unsharp_polymage.cpp:10, fed the
    uint8-quantised image it is written for), pipeline_laplacian
    (sandbox/video_demo/laplacian_polymage.cpp:10);
  - ``reference variant``: pipeline_bilateral (sandbox/video_demo/
    bilateral_polymage.cpp:10), the reference's bilateral grid for uint8
    BGR frames (15 z bins, grey conversion), fed the image as grey BGR;
  - ``restatement``: the camera pipe's C restatement (oracle/campipe.c,
    OpenMP over rows), which equals the reference's spec byte for byte;
  - ``port``: the NumPy FP64 restatement (single-threaded) where the
    reference holds no compiled code (pyramids, interpolation, Jacobi,
    multigrid, NAS MG).
  OpenMP libraries run with ``threads`` threads (libgomp's
  omp_set_num_threads); NumPy ports always use one.
"""

import ctypes
import ctypes.util
import os
import time

import numpy as np

from . import (bilateral as OB, campipe as OC, harris as OH,
               interpolate as OI, jacobi as OJ, laplacian as OL,
               multigrid as OM, nas_mg as ON, pyramid as OP, ref,
               unsharp as OU)

_gomp = None


def set_threads(n):
    """Thread count of the OpenMP runtime the baseline libraries share."""
    global _gomp
    os.environ["OMP_NUM_THREADS"] = str(n)
    if _gomp is None:
        name = ctypes.util.find_library("gomp") or "libgomp.so.1"
        try:
            _gomp = ctypes.CDLL(name)
        except OSError:
            _gomp = False
    if _gomp:
        _gomp.omp_set_num_threads(int(n))


def _cycle_kw(app):
    from polymage_b200.apps import catalog
    kw = catalog._BUILDERS[app][1]
    return dict(L=kw['L'], nu1=kw['nu1'], nu2=kw['nu2'], nuc=kw['nuc'],
                gamma=kw.get('gamma', 1)), kw.get('dims', 2)


def expected(app, params, inputs):
    """({output name: reference array}, {output name: bool mask of the
    points compared, or None for all})."""
    if app == 'harris':
        return {'harris': OH.harris(inputs['img'])}, {'harris': None}
    if app == 'unsharp':
        img = inputs['img']
        t, w = params['threshold'], params['weight']
        R, C = params['R'], params['C']
        ref_ = OU.unsharp(img, t, w)
        ok = np.zeros(ref_.shape, bool)
        xs, ys = OU.defined_region(R, C)
        ok[:, xs, ys] = OU.margin(img, t)[:, xs, ys] > 1e-6
        return {'mask': ref_}, {'mask': ok}
    if app == 'campipe':
        return ({'process': OC.campipe(inputs['img'], params['colour_temp'],
                                       params['contrast'], params['gamma'],
                                       inputs['matrix_3200'],
                                       inputs['matrix_7000'])},
                {'process': None})
    if app == 'bilateral':
        return {'filtered': OB.bilateral(inputs['input'])}, {'filtered': None}
    if app == 'pyramid':
        return ({'blend': OP.pyramid_blend(inputs['img1'], inputs['img2'],
                                           inputs['mask'])},
                {'blend': None})
    if app == 'pyramid8':
        return ({'blend': OP.pyramid_blend_clamped(
            inputs['img1'], inputs['img2'], inputs['mask'], L=8)},
            {'blend': None})
    if app == 'laplacian':
        return ({'laplacian': OL.local_laplacian(
            inputs['img_colour'], params['alpha'], params['beta'])},
            {'laplacian': None})
    if app == 'interpolate':
        return {'interpolate': OI.interpolate(inputs['img'])}, \
            {'interpolate': None}
    if app in ('jacobi2d', 'jacobi3d'):
        from polymage_b200.apps import catalog
        fn = OJ.jacobi2d if app == 'jacobi2d' else OJ.jacobi3d
        T = (catalog.JACOBI2D if app == 'jacobi2d' else catalog.JACOBI3D)['T']
        return {'jacobi': fn(inputs['V_'], inputs['F_'], T=T)}, \
            {'jacobi': None}
    if app in ('vcycle', 'wcycle', 'vcycle3d', 'wcycle3d'):
        kw, dims = _cycle_kw(app)
        fn = OM.v_cycle if dims == 2 else OM.v_cycle3d
        name = {'vcycle': 'Vcycle', 'wcycle': 'Wcycle',
                'vcycle3d': 'Vcycle3d', 'wcycle3d': 'Wcycle3d'}[app]
        return {name: fn(inputs['V_'], inputs['F_'], params['n'], **kw)}, \
            {name: None}
    if app == 'maxfilter':
        from . import maxfilter as OMF
        return {'final': OMF.maxfilter(inputs['img'])}, {'final': None}
    if app == 'nlmeans':
        from . import nlmeans as ONL
        return ({'non_local_means': ONL.nlmeans(
            inputs['img'], params['patch_size'], params['search_area'])},
            {'non_local_means': None})
    if app == 'mg3p':
        from polymage_b200.apps import catalog
        u, r = ON.mg3p(inputs['U'], inputs['V'], inputs['R'],
                       prob_class=catalog.MG3P['prob_class'])
        return {'MG_U': u, 'MG_R': r}, {'MG_U': None, 'MG_R': None}
    raise ValueError(app)


def _runner(app, params, inputs):
    """(kind, description, zero-argument callable running the baseline once,
    OpenMP or not)."""
    if app == 'harris' and ref.available('harris'):
        img = np.ascontiguousarray(inputs['img'], np.float32)
        return ('reference', 'refHarris (reference generated C++)',
                lambda: ref.ref_harris(img), True)
    if app == 'unsharp' and ref.available('unsharp'):
        img = inputs['img']
        u8 = np.ascontiguousarray(np.moveaxis(np.clip(
            img * 255.0, 0, 255).astype(np.uint8), 0, 2))
        R, C = params['R'], params['C']
        out = np.zeros((R, C, 3), np.float32)
        return ('reference', 'pipeline_mask (reference generated C++, uint8 '
                'interleaved input)',
                lambda: ref.ref_unsharp(u8, params['threshold'],
                                        params['weight'], out), True)
    if app == 'laplacian' and ref.available('laplacian'):
        fr = inputs['img_colour']
        out = np.zeros_like(fr)
        return ('reference', 'pipeline_laplacian (reference generated C++)',
                lambda: ref.ref_laplacian(fr, params['alpha'], params['beta'],
                                          out), True)
    if app == 'bilateral' and ref.available('bilateral'):
        img = inputs['input']
        rows, cols = img.shape
        bgr = np.ascontiguousarray(np.repeat(np.clip(
            img * 255.0, 0, 255).astype(np.uint8)[:, :, None], 3, axis=2))
        out = np.zeros((rows, cols), np.float32)
        lib = ref._lib('bilateral')
        fn = lib.pipeline_bilateral
        fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                       ctypes.c_void_p]
        fn.restype = None
        return ('reference variant', 'pipeline_bilateral (reference '
                'generated C++, video-demo variant: uint8 BGR input, 15 z '
                'bins)',
                lambda: fn(cols + 56, rows + 56, bgr.ctypes.data,
                           out.ctypes.data), True)
    if app == 'campipe':
        return ('restatement', 'oracle/campipe.c (C restatement, equal to '
                'the reference spec byte for byte; OpenMP)',
                lambda: OC.campipe(inputs['img'], params['colour_temp'],
                                   params['contrast'], params['gamma'],
                                   inputs['matrix_3200'],
                                   inputs['matrix_7000']), True)
    return ('port', 'NumPy FP64 restatement (single-threaded)',
            lambda: expected(app, params, inputs), False)


def time_baseline(app, params, inputs, threads, budget_s=1.5, max_runs=5):
    """Best wall time of the CPU baseline over up to ``max_runs`` runs
    within ``budget_s`` (at least one run after a warm-up run)."""
    kind, desc, run, omp = _runner(app, params, inputs)
    if not omp:
        threads = 1
    set_threads(threads)
    run()                                   # warm-up
    ts = []
    end = time.perf_counter() + budget_s
    while not ts or (time.perf_counter() < end and len(ts) < max_runs):
        t0 = time.perf_counter()
        run()
        ts.append(time.perf_counter() - t0)
    return {'kind': kind, 'impl': desc, 'cores': threads,
            'seconds': min(ts), 'runs': len(ts)}


def check_and_time(app, params, inputs, threads):
    """(expected outputs, masks, {label: baseline}) for ``app``: a NumPy
    port is timed on the very run that produces the expected outputs (one
    run, one core); compiled baselines are timed separately on ``threads``
    cores and on one."""
    kind = _runner(app, params, inputs)[0]
    if kind == 'port':
        t0 = time.perf_counter()
        exp, masks = expected(app, params, inputs)
        b = {'kind': kind, 'impl': 'NumPy FP64 restatement (single-threaded)',
             'cores': 1, 'seconds': time.perf_counter() - t0, 'runs': 1}
        return exp, masks, {'one_core': b}
    exp, masks = expected(app, params, inputs)
    return exp, masks, {'all_cores': time_baseline(app, params, inputs,
                                                   threads),
                        'one_core': time_baseline(app, params, inputs, 1)}
