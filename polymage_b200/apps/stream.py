"""Serving a mixed stream of requests: Harris, unsharp mask and pyramid
blending on images of uneven sizes, batched per pipeline.

  python -m polymage_b200.apps.stream --requests 1024 --seed 1

The stream is cut into chunks that fit a device-memory budget; within a
chunk the requests of each pipeline go through its batch entry
(``pipeline_<name>_batch``: one launch per group for all of them, a
persistent grid over a device tile queue when the tiles outnumber the
CTAs the GPU holds at once).  Request inputs are created on the device
(U[0,1)); the timed region of a chunk is its batch calls only, bracketed by
CUDA events on the launching stream.

Pyramid requests blend with 8 levels and indices clamped at each level's
borders (``pyramid_blending_clamped``): the reference's spec
(pyramid_blend/polymage_blending.py:24, 4 levels) shrinks its domains by
2^(L+1) pixels per side, which at 8 levels leaves references outside the
domains for every size in the stream.
"""

import argparse
import json

import numpy as np

from . import catalog

KINDS = ("harris", "unsharp", "pyramid8")


def make_stream(n=1024, seed=1, lo=256, hi=4096):
    """``n`` requests (pipeline, rows, cols): pipeline uniform over
    ``KINDS``, sides uniform over lo..hi, from ``seed``."""
    rng = np.random.default_rng(seed)
    kinds = rng.integers(0, len(KINDS), n)
    sides = rng.integers(lo, hi + 1, (n, 2))
    return [(KINDS[k], int(r), int(c)) for k, (r, c) in zip(kinds, sides)]


def request_bytes(kind, r, c):
    """Compulsory bytes of one request (inputs read once, output written
    once) and its output pixels (rows x cols)."""
    if kind == 'harris':
        return 8 * r * c, r * c
    if kind == 'unsharp':
        return 4 * 3 * ((r + 4) * (c + 4) + r * c), r * c
    return 4 * (7 * r * c + 3 * r * c), r * c


def _request_io(kind, r, c, dev, gen):
    import torch

    def rnd(*shape):
        return torch.rand(shape, generator=gen, device=dev)
    if kind == 'harris':
        return ({'R': r - 2, 'C': c - 2}, {'img': rnd(r, c)},
                {'harris': torch.empty((r, c), device=dev)})
    if kind == 'unsharp':
        return ({'R': r, 'C': c, 'threshold': 0.001, 'weight': 3.0},
                {'img': rnd(3, r + 4, c + 4)},
                {'mask': torch.empty((3, r, c), device=dev)})
    return ({'R': r, 'C': c},
            {'img1': rnd(3, r, c), 'img2': rnd(3, r, c), 'mask': rnd(r, c)},
            {'blend': torch.empty((3, r, c), device=dev)})


def serve(reqs, device=None, budget=8 << 30, seed=1, keep=False,
          concurrent=True):
    """Run the stream; returns totals (GPU ms of the batch calls, output
    pixels, compulsory bytes, chunks, batch calls); with ``keep`` also
    every request's (pipeline, params, inputs, outputs).  ``concurrent``:
    the pipelines' batch calls of a chunk run on their own streams, forked
    from the timing stream and joined back into it (they share no data:
    each library has its own workspace); otherwise one after another on
    the timing stream."""
    import torch
    dev = device or torch.device("cuda", torch.cuda.current_device())
    libs = dict((k, catalog.build(k)) for k in KINDS)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    stream = torch.cuda.current_stream(dev)
    side = dict((k, torch.cuda.Stream(dev)) for k in KINDS)
    total_ms, pixels, nbytes, chunks, calls = 0.0, 0, 0, 0, 0
    kept = []
    i = 0
    while i < len(reqs):
        chunk, used = [], 0
        while i < len(reqs):
            b, _ = request_bytes(*reqs[i])
            if chunk and used + b > budget:
                break
            chunk.append(reqs[i])
            used += b
            i += 1
        per = dict((k, ([], [], [])) for k in KINDS)
        for kind, r, c in chunk:
            prm, ins, outs = _request_io(kind, r, c, dev, gen)
            per[kind][0].append(prm)
            per[kind][1].append(ins)
            per[kind][2].append(outs)
            b, px = request_bytes(kind, r, c)
            nbytes += b
            pixels += px
            if keep:
                kept.append((kind, prm, ins, outs))
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for kind in KINDS:
            if not per[kind][0]:
                continue
            s = stream
            if concurrent:
                s = side[kind]
                s.wait_event(e0)
            libs[kind].run_batch(*per[kind], stream=s.cuda_stream)
            if concurrent:
                stream.wait_stream(s)
            calls += 1
        e1.record(stream)
        torch.cuda.synchronize(dev)
        for cp in libs.values():
            cp.check()
        total_ms += e0.elapsed_time(e1)
        chunks += 1
        del per
    out = {"ms": total_ms, "pixels": pixels, "bytes": nbytes,
           "chunks": chunks, "batch_calls": calls}
    if keep:
        out["requests"] = kept
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=1024)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--budget-gb", type=float, default=8.0)
    ap.add_argument("--serial", action="store_true",
                    help="the pipelines' batches one after another")
    args = ap.parse_args()
    reqs = make_stream(args.requests, args.seed)
    serve(reqs, budget=int(args.budget_gb * (1 << 30)), seed=args.seed,
          concurrent=not args.serial)      # sizes workspaces
    r = serve(reqs, budget=int(args.budget_gb * (1 << 30)), seed=args.seed,
              concurrent=not args.serial)
    r["mpix_s"] = r["pixels"] / (r["ms"] / 1e3) / 1e6
    r["gb_s"] = r["bytes"] / (r["ms"] / 1e3) / 1e9
    print(json.dumps(r))


if __name__ == "__main__":
    main()
