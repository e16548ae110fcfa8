#!/usr/bin/env python
"""Benchmark of the PolyMage unsharp-mask pipeline on B200.

Workload (one step): unsharp mask over one 3-channel 4096x4096 float32
image, values U[0,1) from seed 0 with the reference's 2-pixel zero ghost
zone, weight 3, threshold 0.001; one launch of the fused group kernel.

Reported (one JSON line, rank 0):
  value     MPix/s of the whole job with inputs resident in HBM, timed with
            CUDA events over exactly --steps steps (max over ranks)
  e2e       the same metric through the reference's C ABI
            (``pipeline_unsharp`` on pinned host buffers: host->device copy
            of the input and device->host copy of the result every step)
  roofline  compulsory bytes per launch / mean kernel time vs the measured
            HBM copy bandwidth
  cpu_baseline  the reference's own generated C++ (pipeline_mask, OpenMP on
            all host cores) on a bounded sample of the same workload
  clocks    SM clocks and throttle reasons sampled during the timed region
  pipelines every shipped pipeline (the five benchmark configurations, the
            local Laplacian and the widening pipelines) at its benchmark
            size: MPix/s, the compulsory-bytes HBM roofline fraction and the
            spread of its run times (polymage_b200.apps.measure); with the
            cpu_baseline leg also its error against the oracle on the same
            inputs and its CPU baseline on all host cores and on one
            (oracle/baselines.py)

``--impl reference`` times the reference's CPU implementation alone.
Multi-GPU (torchrun): every rank runs its own image (replicas, weak
scaling); no collective is on the data path.
"""

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

R = C = 4096
THRESHOLD, WEIGHT = 0.001, 3.0
IN_BYTES = 3 * (R + 4) * (C + 4) * 4
OUT_BYTES = 3 * R * C * 4
ALG_BYTES = IN_BYTES + OUT_BYTES          # compulsory bytes per step
D2H_BYTES = 3 * (R - 1) * (C - 1) * 4     # points the pipeline writes
METRIC = "MPix/s, unsharp mask 3x4096x4096 float32 (w=3, thr=0.001)"
WORKLOAD = "unsharp_mask 3x4096x4096 float32 w=3 threshold=0.001"


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    return ws, rank


def max_over_ranks(x, device, world_size):
    """The largest of every rank's ``x`` (a time), for whole-job rates."""
    if world_size <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, world_size, seconds):
    """Whole-job throughput: every rank processed ``units_per_rank``."""
    return world_size * units_per_rank / seconds


# ---------------------------------------------------------------------------
class Clocks(object):
    """nvidia-smi sampler running while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,"
         "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                universal_newlines=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [],
                    "samples": 0}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=10)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
def cpu_baseline(budget_s=3.0):
    """The reference's own generated C++ (pipeline_mask from
    sandbox/video_demo/unsharp_polymage.cpp, OpenMP on all host threads) on
    the same image size; its input is the uint8 image it is written for."""
    threads = os.cpu_count()
    os.environ["OMP_NUM_THREADS"] = str(threads)
    import oracle.ref as ref
    if not ref.available("unsharp"):
        return None
    rng = np.random.default_rng(0)
    u8 = rng.integers(0, 256, (R + 4, C + 4, 3), dtype=np.uint8)
    out = np.zeros((R, C, 3), np.float32)
    ref.ref_unsharp(u8, THRESHOLD, WEIGHT, out)       # warm-up
    ts = []
    t_end = time.perf_counter() + budget_s
    while time.perf_counter() < t_end or len(ts) < 3:
        t0 = time.perf_counter()
        ref.ref_unsharp(u8, THRESHOLD, WEIGHT, out)
        ts.append(time.perf_counter() - t0)
    best = min(ts)
    return {"value": R * C / best / 1e6, "unit": "MPix/s", "cores": threads,
            "kind": "reference",
            "sample": "%d full 3x%dx%d images through pipeline_mask "
                      "(reference generated C++, uint8 interleaved input), "
                      "best of %d" % (len(ts), R, C, len(ts))}


def pipeline_check(app, dev):
    """The cpu_baseline leg for one shipped pipeline at its benchmark size:
    its output on the GPU (host-buffer entry) against the oracle on the
    same inputs (``error``), and the CPU baseline timed on all host cores
    and on one (``cpu_baseline``; oracle/baselines.py says which
    implementation each pipeline has)."""
    from polymage_b200.apps import catalog, measure
    import oracle.baselines as OBL
    cp = catalog.build(app)
    prm, host_in, out_spec, pixels, desc = measure.workload(app)
    outs = dict((k, np.zeros(sh, dt)) for k, (sh, dt) in out_spec.items())
    cp.run_host(prm, host_in, outs)
    exp, masks, base = OBL.check_and_time(app, prm, host_in, os.cpu_count())
    err = {}
    for k, ref in exp.items():
        got = outs[k]
        m = masks.get(k)
        integer = np.issubdtype(got.dtype, np.integer)
        d = np.abs(got.astype(np.float64) - np.asarray(ref, np.float64))
        scale = float(np.abs(ref).max()) or 1.0
        sel = d if m is None else d[m]
        e = {"max_abs": float(sel.max()),
             "max_abs_over_max_ref": float(sel.max()) / scale}
        if integer:
            e["mismatched"] = int(np.count_nonzero(sel))
            e["of"] = int(sel.size)
        else:
            r = np.abs(np.asarray(ref, np.float64))
            rel = d / np.maximum(r, 1e-6 * scale)
            e["max_rel_floor_1e-6"] = float((rel if m is None else
                                             rel[m]).max())
        if m is not None:
            e["tie_band_excluded"] = int(m.size - np.count_nonzero(m))
        err[k] = e
    for b in base.values():
        b["value"] = pixels / b["seconds"] / 1e6
        b["unit"] = "MPix/s"
    return {"error": err, "cpu_baseline": base}


def learned_vs_exhaustive():
    """The learned tuner replayed on the committed B200 timing database
    (polymage_b200/data/timing_db_b200.jsonl: every configuration of the
    reference's search space, measured): per pipeline, the cost model is
    trained on the GPU by this package's kernels on the other pipelines'
    rows only, picks 8 configurations, and its best pick's time is
    compared with the database's best (the exhaustive result)."""
    from polymage_b200 import costmodel, tuner
    rows = tuner.load_db(costmodel.DB_PATH)
    out = {}
    for app in sorted(set(r['app'] for r in rows)):
        t0 = time.time()
        ratio, n, uniq = costmodel.evaluate_on_db(rows, app, batches=(8,),
                                                  seed=0)
        out[app] = {"learned_over_exhaustive_time": ratio, "timed": n,
                    "distinct_plans": uniq,
                    "replay_s": time.time() - t0}
    return out


def int_roofline(entry, int_peak):
    """Integer-ALU roofline of the camera pipe: its kernel's integer
    thread instructions per image (one ncu count of the default build,
    profiles/counters.json) over the pipeline time, against the measured
    integer throughput (polymage_b200.apps.measure.int_peak)."""
    p = os.path.join(ROOT, "profiles", "counters.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f).get("campipe")
    if not d:
        return None
    rate = d["integer_thread_inst"] / (entry["ms"] / 1e3)
    peak = max(v["thread_inst_per_s"] for v in int_peak.values())
    return {"integer_thread_inst_per_image": d["integer_thread_inst"],
            "achieved_per_s": rate, "peak_per_s": peak,
            "frac": rate / peak, "counted_on": d.get("kernel")}


def run_reference_arm(args):
    ws, rank = _dist()
    if rank != 0:
        return 0
    threads = os.cpu_count()
    os.environ["OMP_NUM_THREADS"] = str(threads)
    import oracle.ref as ref
    if not ref.available("unsharp"):
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libref_unsharp.so not built"}))
        return 0
    # each step: one full 3x4096x4096 image, as in this arm's own steps
    # (about 8 ms on 16 host cores, so a run of a few thousand steps still
    # ends within a minute or two)
    rng = np.random.default_rng(0)
    u8 = rng.integers(0, 256, (R + 4, C + 4, 3), dtype=np.uint8)
    out = np.zeros((R, C, 3), np.float32)
    for _ in range(args.warmup):
        ref.ref_unsharp(u8, THRESHOLD, WEIGHT, out)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ref.ref_unsharp(u8, THRESHOLD, WEIGHT, out)
    dt = time.perf_counter() - t0
    v = args.steps * R * C / dt / 1e6
    line = {"metric": METRIC, "value": v, "unit": "MPix/s", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic uint8 U{0..255} (the reference variant's "
                    "input type), seed 0",
            "config": {"workload": WORKLOAD, "sample": "one 3x%dx%d image "
                       "per step" % (R, C)},
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "MPix/s", "cores": threads,
                             "kind": "reference",
                             "sample": "%d steps of a 3x%dx%d image "
                                       "through pipeline_mask" % (
                                           args.steps, R, C)},
            "e2e": {"value": v, "unit": "MPix/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
def _load_traffic(kernel):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    v = d.get(kernel)
    return float(v["bytes_per_launch"]) if v else None


def run(args):
    import torch
    import torch.distributed as dist
    ws, rank = _dist()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=dev)
    from polymage_b200.apps.unsharp_mask import build_unsharp
    import oracle.unsharp as OU

    from polymage_b200.apps import catalog
    cp = build_unsharp(**catalog.UNSHARP).build()
    kernel = cp.module.meta['groups'][0]['kernel']
    prm = {'R': R, 'C': C, 'threshold': THRESHOLD, 'weight': WEIGHT}
    host_in = OU.make_input(R, C, seed=0)
    d_in = torch.from_numpy(host_in).to(dev)
    d_out = torch.zeros((3, R, C), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        cp.run_dev(prm, {'img': d_in}, {'mask': d_out},
                   stream=stream.cuda_stream)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize(dev)
    cp.check()

    # --- timed region: exactly --steps steps, inputs resident in HBM -------
    clocks = Clocks(torch.cuda.current_device()) if rank == 0 else None
    if clocks:
        clocks.start()
        time.sleep(0.3)
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for i in range(args.steps):
        ev[i][0].record(stream)
        step()
        ev[i][1].record(stream)
    t1.record(stream)
    torch.cuda.synchronize(dev)
    if ws > 1:
        dist.barrier()
    clk = clocks.stop() if clocks else None
    cp.check()
    elapsed_ms = t0.elapsed_time(t1)
    per_step = sorted(a.elapsed_time(b) for a, b in ev)
    kern_ms = float(np.mean(per_step))
    elapsed_ms = max_over_ranks(elapsed_ms, dev, ws)
    value = job_rate(args.steps * R * C, ws, elapsed_ms / 1e3) / 1e6

    # --- end to end through the reference C ABI (host buffers) -------------
    pin_in = torch.empty(host_in.shape, dtype=torch.float32,
                         pin_memory=True)
    pin_in.numpy()[...] = host_in
    pin_out = torch.zeros((3, R, C), dtype=torch.float32, pin_memory=True)
    a_in, a_out = pin_in.numpy(), pin_out.numpy()
    e2e_steps = max(3, min(args.steps, 20))
    for _ in range(2):
        cp.run_host(prm, {'img': a_in}, {'mask': a_out})
    if ws > 1:
        dist.barrier()
    s0 = time.perf_counter()
    for _ in range(e2e_steps):
        cp.run_host(prm, {'img': a_in}, {'mask': a_out})
    e2e_s = time.perf_counter() - s0
    e2e_s = max_over_ranks(e2e_s, dev, ws)
    e2e = job_rate(e2e_steps * R * C, ws, e2e_s) / 1e6

    if rank == 0:
        peak, peak_kind = _peaks()
        achieved = ALG_BYTES / (kern_ms / 1e3) / 1e9
        traffic = _load_traffic(kernel)
        line = {
            "metric": METRIC, "value": value, "unit": "MPix/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": elapsed_ms / args.steps,
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: U[0,1) seed 0, 2-px zero ghost zone",
            "config": {"workload": WORKLOAD,
                       "tile": list(catalog.UNSHARP["tile_sizes"]),
                       "options": list(catalog.UNSHARP["options"]),
                       "kernel": kernel,
                       "l2": "inputs larger than L2 (201.7 MB in + 201.3 MB "
                             "out per step vs 126 MB L2)",
                       "parallelism": "replicas x%d" % ws},
            "e2e": {"value": e2e, "unit": "MPix/s",
                    "h2d_bytes_per_step": IN_BYTES,
                    "d2h_bytes_per_step": D2H_BYTES,
                    "api": "pipeline_unsharp (host buffers, synchronous)"},
            "roofline": {"bound": "hbm", "achieved": achieved,
                         "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": peak_kind,
                         "alg_bytes_per_launch": ALG_BYTES,
                         "kernel_ms": kern_ms,
                         "kernel_ms_min": per_step[0],
                         "kernel_ms_median": float(np.median(per_step)),
                         "kernel_ms_max": per_step[-1]},
            "gpu_launches": args.steps,
            "clocks": clk,
        }
        if not args.no_pipelines:
            # every shipped pipeline at its benchmark size (device buffers,
            # L2 flushed before each run): MPix/s and compulsory-bytes
            # roofline fraction
            from polymage_b200.apps import measure
            line["pipelines"] = dict(
                (a, measure.measure(a, steps=50, warmup=5, device=dev))
                for a in measure.APPS + measure.WIDENING)
            line["pipelines"]["bilateral_batch64"] = \
                measure.measure_bilateral_batch(64, device=dev)
            line["pipelines"]["stream1024"] = measure.measure_stream(
                1024, device=dev)
            ip = measure.int_peak(device=dev)
            line["int_peak"] = ip
            ir = int_roofline(line["pipelines"]["campipe"], ip)
            if ir:
                line["pipelines"]["campipe"]["int_roofline"] = ir
            line["learned_vs_exhaustive"] = learned_vs_exhaustive()
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline()
            if "pipelines" in line:
                for app, entry in line["pipelines"].items():
                    if app in measure.APPS + measure.WIDENING:
                        entry.update(pipeline_check(app, dev))
        print(json.dumps(line))
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="polymage_b200",
                    choices=["polymage_b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-pipelines", action="store_true",
                    help="skip the per-pipeline throughput table")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    return run(args)


if __name__ == "__main__":
    sys.exit(main())
