#!/usr/bin/env python
"""Benchmark: N4 volumes/s to CV < 1e-3 at 256x256x176 on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B] [--impl ours|reference]

One step = one batch of B synthetic 256x256x176 phantoms (shrink 4, 4 levels,
<= 50 iterations per level, convergence 0.001, 200 bins, FWHM 0.15, Wiener
0.01) bias-corrected to convergence: the masked log volumes are pooled to
32x32x24, the learned encoder predicts every volume's first-level lattice,
and the batch runs as persistent cluster launches with those warm lattices
(overlapped sub-batches: each sub-batch's prologue, warm start and correction
run beside the other sub-batches' N4 launches), recorded once as a CUDA graph
(``n4_batch_graph_*``) and replayed.  The cluster size of the batch is chosen
by the autotuner (``n4_autotune``, untimed, before the warm-up).  ``value`` is whole-job volumes/s of that
batched + warm-started path with the inputs resident in HBM.  Beside it:
``batched_plain`` (the same graph without warm start), ``batched_without_graph``
(``n4_run_batched`` at every step), ``plain`` (``n4_run``, one volume per
call: the single-volume path the batched one is compared with), and ``e2e``
(the same warm-started batched correction through ``n4_run_batched_host``:
images and float masks in pinned host memory, corrected volumes and lattices
back into pinned host memory, the library overlapping the uploads, runs and
downloads of sub-batches of 8 volumes; its device time runs from the first
upload to the last download of every step).

Multi-GPU: one process per GPU (torchrun); volumes are independent, so each
rank corrects its own batch (replicas, weak scaling, no collective on the data
path); the timed region is bracketed by barriers and the time is the maximum
over ranks.

``--impl reference`` times the reference algorithm on the host cores: the
FP64 restatement of N4.py in ``oracle/`` (N4.py itself cannot run here: its
per-voxel Python loops take ~3 minutes per volume), one volume per process
on every available core.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cuda-n4_b200"))

METRIC = "N4 volumes/s to CV<1e-3 at 256²×176, batched+warm-start vs plain; fit GB/s"
SHAPE = (256, 256, 176)
GEN = dict(sigma=0.02, grid=6, coeff_std=0.25)
SHRINK, LEVELS, ITERS, THR = 4, 4, 50, 0.001
# per-iteration algorithmic bytes per fitting voxel of an HBM-streaming N4
# iteration: fit 5 (logU 4 + mask 1) + histogram 5 + evaluate/CV/update 17
ITER_BYTES_PER_VOXEL = 27
# final correction: read im 4 + write corrected 4 per full-resolution voxel
CORRECT_BYTES_PER_VOXEL = 8
# DRAM bytes (read + write) of one k_n4_cluster launch per volume of this
# workload, from an ncu capture of a 4-volume launch (3.323 MB read, nothing
# written): the volume stays in shared memory, so only its initial load moves
TRAFFIC_PER_VOLUME = 3.323392e6 / 4


def workload_desc(batch):
    return dict(workload="c2: 256x256x176 float32 phantoms, shrink 4 -> 64x64x44, 4 levels, <=50 it/level, "
                         "CV<0.001, 200 bins, FWHM 0.15, Wiener 0.01, low_value 0",
                batch_per_gpu=batch, parallelism="replicas (volume-parallel)",
                l2="inputs larger than L2: each step reads B distinct volumes (B x 92 MB)")


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """Samples SM clocks and throttle reasons every 20 ms (NVML)."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, index):
        self.index = index
        self.samples, self.reasons = [], set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
        except Exception:
            return self

        def run():
            while not self._stop.is_set():
                try:
                    self.samples.append(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
                    r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                    for bit, name in self.REASONS.items():
                        if r & bit:
                            self.reasons.add(name)
                except Exception:
                    pass
                self._stop.wait(0.02)

        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()
        return self

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join()
        s = sorted(self.samples)
        med = s[len(s) // 2] if s else None
        return {"sm_mhz": med, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(s)}


# ---------------------------------------------------------------- reference arm
def _ref_init(seed):
    global _REF_VOL
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from n4b200.phantom import make_phantom
    ph = make_phantom(SHAPE, seed=seed, **GEN)
    _REF_VOL = (ph.im, ph.mask)


def _ref_one(_):
    import n4_oracle as O
    im, mask = _REF_VOL
    rep = {}
    O.N4Shrink(im, mask, SHRINK, low_value=0, maximumNumberOfLevels=LEVELS,
               maximumNumberOfIterations=[ITERS] * LEVELS, ConvergenceThreshold=THR, report=rep)
    return sum(rep["iterations"])


def run_reference(args, rank):
    if rank != 0:
        return 0
    import multiprocessing as mp
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[k] = "1"
    cores = min(os.cpu_count() or 1, 64)
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores, initializer=_ref_init, initargs=(7,)) as pool:
        for _ in range(args.warmup):
            pool.map(_ref_one, range(cores))
        t0 = time.perf_counter()
        iters = []
        for _ in range(args.steps):
            iters += pool.map(_ref_one, range(cores))
        dt = time.perf_counter() - t0
    value = cores * args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "volumes/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * dt / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload_desc(cores),
        "cpu_baseline": {"value": value, "unit": "volumes/s", "cores": cores, "kind": "port",
                         "sample": f"each step: {cores} phantoms, one per process, FP64 numpy restatement "
                                   f"of N4.py run to convergence (mean {sum(iters) / len(iters):.1f} iterations)"},
        "e2e": {"value": value, "unit": "volumes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline_single(seconds=12.0):
    """The oracle on one host core over a bounded sample (whole volumes)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import n4_oracle as O
    from n4b200.phantom import make_phantom
    n, t_total, iters = 0, 0.0, 0
    while t_total < seconds and n < 32:
        ph = make_phantom(SHAPE, seed=500 + n, **GEN)
        rep = {}
        t0 = time.perf_counter()
        O.N4Shrink(ph.im, ph.mask, SHRINK, low_value=0, maximumNumberOfLevels=LEVELS,
                   maximumNumberOfIterations=[ITERS] * LEVELS, ConvergenceThreshold=THR, report=rep)
        t_total += time.perf_counter() - t0
        iters += sum(rep["iterations"])
        n += 1
    return {"value": n / t_total, "unit": "volumes/s", "cores": 1, "kind": "port",
            "sample": f"{n} phantoms 256x256x176 corrected to convergence by the FP64 restatement of N4.py "
                      f"on one core ({iters / n:.1f} iterations per volume, phantom generation untimed)"}


def measure_components(dev, ctx, hbm_peak, reps=10):
    """Standalone HBM-bound kernels at the 512x512x320 scale: the fit's z
    contraction (k_fit_rows_v5) on the 256x256x160 fitting grid (reads field
    4 B + float mask 4 B per voxel) and the dense evaluation (k_correct) at
    full resolution (writes 4 B per voxel); device time of the kernel alone
    from the library's stage events, mean of `reps` calls, L2 evicted before
    each."""
    import numpy as np
    import torch
    import n4b200
    gen = torch.Generator(device=dev).manual_seed(5)
    fit_shape, full_shape = (256, 256, 160), (512, 512, 320)
    field = torch.randn(fit_shape, device=dev, generator=gen)
    fmask = (torch.rand(fit_shape, device=dev, generator=gen) > 0.4).float()
    lat11 = torch.randn((11, 11, 11), device=dev, generator=gen) * 0.1

    # L2 eviction before every timed call: reading a 256 MB buffer (twice the
    # L2) leaves only its clean lines there, so the timed kernel neither hits
    # its own inputs in L2 nor pays for writing back a flush's dirty lines
    flush = torch.zeros(64 << 20, dtype=torch.float32, device=dev)

    # tile shapes chosen by the component autotuner for these two sizes
    tune_fit = n4b200.autotune_components(field, fmask, (11, 11, 11), ctx=ctx)
    big = torch.randn(full_shape, device=dev, generator=gen)
    tune_eval = n4b200.autotune_components(big, None, (11, 11, 11), ctx=ctx)
    del big

    def kernel_ms(fn, stage):
        fn()
        ctx.set_profiling(True)
        tot = 0.0
        for _ in range(reps):
            flush.sum()
            fn()
            tot += ctx.last_timings()["stage_ms"][stage]
        tm = ctx.last_timings()
        ctx.set_profiling(False)
        return tot / reps, tm
    ms_fit, tf = kernel_ms(lambda: n4b200.FitBspline3D(field, fmask, (11, 11, 11), ctx=ctx), 0)
    ms_eval, te = kernel_ms(lambda: n4b200.EvaluateBspline3D(lat11, (11, 11, 11), full_shape, ctx=ctx), 1)
    nfit, nfull = field.numel(), int(np.prod(full_shape))
    del field, fmask, flush
    fit = 8 * nfit / (ms_fit / 1000) / 1e9
    ups = 4 * nfull / (ms_eval / 1000) / 1e9
    return {
        "fit_gbs": {"value": fit, "frac": fit / hbm_peak, "ms": ms_fit,
                    "shape": {"step_voxels": tf["fit_step"], "steps_in_flight": tf["fit_depth"],
                              "rows_per_cta": tf["fit_rows"]},
                    "tuner_candidates_ms": tune_fit["fit"],
                    "workload": "FitBspline3D z-contraction pass (k_fit_rows_v5) over a 256x256x160 field + "
                                "float mask, 11^3 lattice (8 B per voxel read; L2 evicted before each call)"},
        "upsample_gbs": {"value": ups, "frac": ups / hbm_peak, "ms": ms_eval,
                         "shape": {"rows_per_tile": te["correct_rows"], "threads": te["correct_threads"]},
                         "tuner_candidates_ms": tune_eval["evaluate"],
                         "workload": "EvaluateBspline3D dense evaluation (k_correct) of an 11^3 lattice at "
                                     "512x512x320 (4 B per voxel written)"},
    }


def measure_c3(dev, ctx, reps=2):
    """One 512x512x320 volume (0.5 mm phantom, 8^3-grid bias N(0, 0.25^2),
    Rician 0.02) through n4_run at shrink 2 (256x256x160 fitting grid, the
    whole-GPU path), 4 levels, <= 50 iterations, convergence 0.001."""
    import torch
    import n4b200
    from n4b200.warmstart import phantoms_gpu
    im, mk = phantoms_gpu(1, (512, 512, 320), seed=77, sigma=0.02, grid=8, coeff_std=0.25, device=dev)
    p = n4b200.N4Param(NumberOfFittingLevels=4, MaximumNumberOfIterations=50, ConvergenceThreshold=0.001,
                       low_value=0.0, ShrinkFactor=2)
    res = n4b200.N4(im[0], mk[0], p, ctx=ctx)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record()
    for _ in range(reps):
        n4b200.N4(im[0], mk[0], p, ctx=ctx, synchronous=False)
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / reps
    # stage times of one run (library events on the launching stream)
    ctx.set_profiling(True)
    n4b200.N4(im[0], mk[0], p, ctx=ctx)
    t = ctx.last_timings()
    ctx.set_profiling(False)
    st = dict(zip(("prologue", "n4_levels_iterations", "tables", "correction"), t["stage_ms"]))
    full = t["full_voxels"]
    return {"workload": "512x512x320 float32 phantom, shrink 2 -> 256x256x160, 4 levels, <=50 it/level, CV<0.001",
            "ms_per_volume": ms, "volumes_per_s": 1000.0 / ms, "iterations": res.report["iterations"][:4],
            "path": res.report["path"], "ctas": res.report["cluster_size"], "stages_ms": st,
            "prologue_gbs": (8 * full + 4 * t["fit_voxels"]) / (st["prologue"] / 1000.0) / 1e9,
            "correction_gbs": 8 * full / (st["correction"] / 1000.0) / 1e9}


def schedule_summary(reports, fit_voxels):
    """How a batched run used its clusters, from the per-volume device
    timestamps of the reports: a persistent cluster keeps its SMs, so the SM
    of a volume's leading CTA names its cluster.  makespan = first begin to
    last end; per cluster, busy = sum of its volumes' times; tail = makespan
    minus the mean cluster finish (the time clusters sit idle at the end on
    average); ns_per_voxel_iteration relates each volume's time to its work."""
    import numpy as np
    rs = [r for r in reports if r.get("device_end_ns")]
    if not rs:
        return {}
    t0 = min(r["device_begin_ns"] for r in rs)
    t1 = max(r["device_end_ns"] for r in rs)
    by = {}
    for r in rs:
        by.setdefault(r["sm"], []).append(r)
    fin = [max(r["device_end_ns"] for r in v) - t0 for v in by.values()]
    busy = [sum(r["device_end_ns"] - r["device_begin_ns"] for r in v) for v in by.values()]
    work = np.array([fv * sum(r["iterations"][:r["levels"]]) for r, fv in zip(reports, fit_voxels)
                     if r.get("device_end_ns")], dtype=np.float64)
    dur = np.array([r["device_end_ns"] - r["device_begin_ns"] for r in rs], dtype=np.float64)
    return {"clusters": len(by), "makespan_ms": (t1 - t0) / 1e6, "mean_cluster_finish_ms": float(np.mean(fin)) / 1e6,
            "mean_cluster_busy_ms": float(np.mean(busy)) / 1e6, "max_cluster_busy_ms": float(np.max(busy)) / 1e6,
            "tail_ms": ((t1 - t0) - float(np.mean(fin))) / 1e6,
            "volume_ms_min_median_max": [float(np.min(dur)) / 1e6, float(np.median(dur)) / 1e6,
                                         float(np.max(dur)) / 1e6],
            "ns_per_voxel_iteration_median": float(np.median(dur / np.maximum(work, 1.0)))}


def measure_c4(dev, enc, n=48, reps=5):
    """48 phantoms with every axis drawn from 96, 104, ..., 288 (4^3-grid bias
    N(0, 0.15^2), Rician 0.03), shrink 4, 4 levels, <= 50 iterations,
    convergence 0.001: the batch with and without the learned warm start,
    after autotuning it (cluster sizes, sub-batches and their per-sub-batch
    cluster sizes), recorded as a graph and replayed, and called eagerly."""
    import numpy as np
    import torch
    import n4b200
    from n4b200.phantom import batch_dims
    from n4b200.warmstart import phantoms_gpu
    vols = []
    for i, sh in enumerate(batch_dims(n, seed=2024)):
        im, mk = phantoms_gpu(1, sh, seed=3000 + i, sigma=0.03, grid=4, coeff_std=0.15, device=dev)
        vols.append((im[0], mk[0]))
    p = n4b200.N4Param(NumberOfFittingLevels=4, MaximumNumberOfIterations=50, ConvergenceThreshold=0.001,
                       low_value=0.0, ShrinkFactor=4)
    ctx = n4b200.Context(dev.index or 0)
    tune = n4b200.autotune(vols, p, ctx=ctx)
    out = {"workload": f"{n} phantoms, axes uniform in 96..288 step 8, shrink 4, 4 levels, <=50 it/level, CV<0.001",
           "autotune": tune}
    def median_ms(fn):
        times = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize(dev)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize(dev)
            times.append(e0.elapsed_time(e1))
        return sorted(times)[len(times) // 2], times

    for name, kw in (("plain", {}), ("warm", {"encoder": enc})):
        for _ in range(2):
            res = n4b200.N4Batch(vols, p, ctx=ctx, **kw)
        # the batch recorded as a graph and replayed (as the headline measures
        # its batch), and n4_run_batched called eagerly (host planning and
        # descriptor upload inside the timed region)
        g = n4b200.N4BatchGraph(vols, p, ctx=ctx, **kw)
        g.launch()
        g.sync()
        ms, times = median_ms(g.launch)
        g.sync()
        g.close()
        ms_eager, _ = median_ms(lambda: n4b200.N4Batch(vols, p, ctx=ctx, synchronous=False, **kw))
        fv = [int(np.prod(n4b200.fitting_dims(p, tuple(im.shape)))) for im, _ in vols]
        out[name] = {"volumes_per_s": n * 1000.0 / ms, "ms_per_batch_median": ms, "ms_per_batch_all": times,
                     "eager_volumes_per_s": n * 1000.0 / ms_eager, "eager_ms_per_batch_median": ms_eager,
                     "iterations_per_volume": sum(sum(r.report["iterations"][:r.report["levels"]]) for r in res) / n,
                     "cluster_sizes": sorted({r.report["cluster_size"] for r in res}),
                     "paths": {k: sum(1 for r in res if r.report["path"] == k) for k in ("cluster", "grid")},
                     "schedule": schedule_summary([r.report for r in res], fv)}
    ctx.close()
    return out


# ---------------------------------------------------------------- our arm
def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    import n4b200
    from n4b200.phantom import make_phantom

    from n4b200.replicas import Replicas, volume_seeds

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    rep = Replicas(world, dev)
    B = args.batch
    vols_host, vols_dev = [], []
    for seed in volume_seeds(rank, B):
        ph = make_phantom(SHAPE, seed=seed, **GEN)
        im_h = torch.from_numpy(ph.im).pin_memory()
        mk_h = torch.from_numpy(ph.mask).pin_memory()
        vols_host.append((im_h, mk_h))
        vols_dev.append((im_h.to(dev), mk_h.to(dev)))
    p = n4b200.N4Param(NumberOfFittingLevels=LEVELS, MaximumNumberOfIterations=ITERS,
                       ConvergenceThreshold=THR, low_value=0.0, ShrinkFactor=SHRINK)
    ctx = n4b200.Context(local_rank)
    stream = torch.cuda.current_stream(dev)

    barrier = rep.barrier
    max_over_ranks = rep.max_over_ranks

    def step_batched():
        return n4b200.N4Batch(vols_dev, p, ctx=ctx, synchronous=False)

    # ---- autotuning (untimed): the cluster size of this batch, recorded in
    # the contexts that run it
    from n4b200.warmstart import load_encoder
    gctx = n4b200.Context(local_rank)
    tune = n4b200.autotune(vols_dev, p, ctx=gctx)
    n4b200.autotune(vols_dev, p, ctx=ctx)

    # ---- headline: prologue -> pooled fitting grids -> encoder -> warm
    # lattices -> batched N4 -> correction, one graph replayed every step
    enc = load_encoder(max_batch=max(B, 1))
    warm = n4b200.N4BatchGraph(vols_dev, p, ctx=gctx, encoder=enc)
    for _ in range(args.warmup):
        warm.launch()
    res_w = warm.sync()
    assert all(r.report["status"] == "N4_OK" for r in res_w), [r.report for r in res_w]
    clocks = ClockSampler(local_rank).start()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        warm.launch()
    e1.record(stream)
    barrier()
    clk = clocks.stop()
    res_w = warm.sync()
    ms = max_over_ranks(e0.elapsed_time(e1))
    value = world * B * args.steps / (ms / 1000.0)
    iters_w = [sum(r.report["iterations"][:r.report["levels"]]) for r in res_w]
    kept = sum(r.report["warm_start_used"] for r in res_w) / B
    lat_w = [r.lattice.clone() for r in res_w]

    # ---- the same batch without warm start (graph replay)
    gctx2 = n4b200.Context(local_rank)
    n4b200.autotune(vols_dev, p, ctx=gctx2)
    graph = n4b200.N4BatchGraph(vols_dev, p, ctx=gctx2)
    for _ in range(args.warmup):
        graph.launch()
    res = graph.sync()
    iters = [sum(r.report["iterations"][:r.report["levels"]]) for r in res]
    assert all(r.report["status"] == "N4_OK" for r in res), [r.report for r in res]
    barrier()
    e0.record(stream)
    for _ in range(args.steps):
        graph.launch()
    e1.record(stream)
    barrier()
    graph.sync()
    ms_gplain = max_over_ranks(e0.elapsed_time(e1))
    # warm-started vs plain: log-bias difference at full resolution over the
    # mask, as it is (raw) and without its mean (a constant log bias is a
    # global intensity scale that the convergence measure std/mean of
    # exp(change) does not see, so N4 never corrects it)
    dims = n4b200.lattice_dims(p)
    draw, dcent = [], []
    for i, r in enumerate(res):
        d = n4b200.EvaluateBspline3D(lat_w[i] - r.lattice, dims, SHAPE, ctx=ctx)
        inside = d[vols_dev[i][1] != 0]
        draw.append(float(inside.abs().max()))
        dcent.append(float((inside - inside.double().mean().float()).abs().max()))
    graph.close()
    warm.close()

    # ---- the same batch through n4_run_batched at every step (host planning
    # and descriptor upload included)
    for _ in range(args.warmup):
        step_batched()
    barrier()
    e0.record(stream)
    h0 = time.perf_counter()
    for _ in range(args.steps):
        step_batched()
    host_ms = 1000 * (time.perf_counter() - h0) / args.steps
    e1.record(stream)
    barrier()
    ms_nograph = max_over_ranks(e0.elapsed_time(e1))

    # ---- stage times of one batched run (events recorded by the library on
    # the launching stream); the warm-started run's stage 0 includes the
    # pooling and the encoder
    ctx.set_profiling(True)
    n4b200.N4Batch(vols_dev, p, ctx=ctx, synchronous=False, encoder=enc)
    t_w = ctx.last_timings()
    step_batched()
    t = ctx.last_timings()
    ctx.set_profiling(False)
    st_ms = t["stage_ms"]          # prologue, N4 levels/iterations, tables, correction
    total_iters = sum(iters)       # plain run: the roofline basis below
    n4_bytes = ITER_BYTES_PER_VOXEL * t["fit_voxels"] / B * total_iters
    achieved = n4_bytes / (st_ms[1] / 1000.0) / 1e9
    hbm_peak, peak_kind = peaks()
    corr_gbs = CORRECT_BYTES_PER_VOXEL * t["full_voxels"] / (st_ms[3] / 1000.0) / 1e9
    pro_gbs = (8 * t["full_voxels"] + 4 * t["fit_voxels"]) / (st_ms[0] / 1000.0) / 1e9

    # ---- plain single-volume path (n4_run, one volume per call)
    for _ in range(args.warmup):
        n4b200.N4(*vols_dev[0], p, ctx=ctx, synchronous=False)
    barrier()
    e0.record(stream)
    for _ in range(args.steps):
        for im, mk in vols_dev:
            n4b200.N4(im, mk, p, ctx=ctx, synchronous=False)
    e1.record(stream)
    barrier()
    ms_plain = max_over_ranks(e0.elapsed_time(e1))
    plain = world * B * args.steps / (ms_plain / 1000.0)

    # ---- end to end through n4_run_batched_host: pinned host inputs ->
    # staging -> batched N4 (warm start) -> pinned host outputs, uploads,
    # runs and downloads of its sub-batches overlapped by the library; the
    # device time of each call runs from its first upload to its last download
    out_h = [torch.empty(a.shape, dtype=torch.float32).pin_memory() for a, _ in vols_host]
    lat_h = [torch.empty(n4b200.lattice_dims(p), dtype=torch.float32).pin_memory() for _ in vols_host]
    hctx = n4b200.Context(local_rank)
    henc = load_encoder(max_batch=16)

    def time_e2e(host):
        outs = list(zip(out_h, lat_h))
        for _ in range(min(args.warmup, 2)):
            n4b200.N4BatchHost(host, p, encoder=henc, outputs=outs, ctx=hctx, device=local_rank)
        barrier()
        tot = 0.0
        w0 = time.perf_counter()
        for _ in range(args.steps):
            res_h, dms = n4b200.N4BatchHost(host, p, encoder=henc, outputs=outs, ctx=hctx, device=local_rank)
            tot += dms
        wall = (time.perf_counter() - w0) * 1000.0
        assert all(r.report["status"] == "N4_OK" for r in res_h)
        barrier()
        return max_over_ranks(tot), wall

    # the host link on this box: pinned H2D, D2H and both at once (8 volumes each way)
    def link_gbs():
        src = [a for a, _ in vols_host[:8]]
        dst = [torch.empty(a.shape, device=dev) for a in src]
        back = [torch.empty(a.shape, dtype=torch.float32).pin_memory() for a in src]
        nbytes = sum(a.numel() * 4 for a in src)
        s_up, s_dn = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

        def timed(up, down):
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            for _ in range(3):
                if up:
                    with torch.cuda.stream(s_up):
                        for a, d in zip(src, dst):
                            d.copy_(a, non_blocking=True)
                if down:
                    with torch.cuda.stream(s_dn):
                        for d, b in zip(dst, back):
                            b.copy_(d, non_blocking=True)
            torch.cuda.synchronize(dev)
            return 3 * nbytes * (int(up) + int(down)) / (time.perf_counter() - t0) / 1e9
        timed(True, False)
        r = {"h2d": timed(True, False), "d2h": timed(False, True), "both_ways": timed(True, True)}
        del dst, back
        return r

    link = link_gbs()
    ms_e2e, wall_e2e = time_e2e(vols_host)
    # the same with byte masks (N4_FLAG_MASK_U8): 1 B instead of 4 B per mask voxel over PCIe
    host_u8 = [(ih, (mh != 0).to(torch.uint8).pin_memory()) for ih, mh in vols_host]
    ms_e2e_u8, wall_e2e_u8 = time_e2e(host_u8)
    h2d_u8 = sum(a.numel() * 4 + b.numel() for a, b in host_u8)
    h2d = sum(a.numel() * 4 + b.numel() * 4 for a, b in vols_host)
    d2h = sum(o.numel() * 4 for o in out_h) + sum(l.numel() * 4 for l in lat_h)

    def link_bound(h2d_bytes):
        # no schedule moves the step's bytes faster than the link: each
        # direction at its one-way rate, both together at the both-ways rate
        t = max(h2d_bytes / link["h2d"], d2h / link["d2h"], (h2d_bytes + d2h) / link["both_ways"]) / 1e9
        return B / t

    comp = measure_components(dev, ctx, peaks()[0])
    c3 = measure_c3(dev, ctx)
    c4 = measure_c4(dev, enc)

    line = {
        "metric": METRIC, "value": value, "unit": "volumes/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_desc(B),
        "roofline": {
            "bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
            "frac": achieved / hbm_peak, "traffic": TRAFFIC_PER_VOLUME * B,
            "traffic_basis": "ncu dram__bytes_read.sum + dram__bytes_write.sum of a 4-volume launch, scaled to "
                             "the batch (grows in proportion: one load of each fitting grid)",
            "kernel": "k_n4_cluster (all levels/iterations of a batch)",
            "basis": f"{ITER_BYTES_PER_VOXEL} B per fitting voxel per iteration "
                     f"(fit 5 + histogram 5 + evaluate/CV/update 17) x iterations / kernel time; "
                     f"peak {peak_kind}",
        },
        "e2e": {"value": world * B * args.steps / (ms_e2e / 1000.0), "unit": "volumes/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "path": "n4_run_batched_host (float masks, warm start, sub-batches of 8 on 4 lanes)",
                "wall_ms_per_step": wall_e2e / args.steps, "link_gbs": link,
                "link_bound_volumes_per_s": world * link_bound(h2d)},
        "e2e_byte_masks": {"value": world * B * args.steps / (ms_e2e_u8 / 1000.0), "unit": "volumes/s",
                           "h2d_bytes_per_step": h2d_u8, "d2h_bytes_per_step": d2h,
                           "path": "same as e2e with uint8 masks (N4_FLAG_MASK_U8)",
                           "wall_ms_per_step": wall_e2e_u8 / args.steps,
                           "link_bound_volumes_per_s": world * link_bound(h2d_u8)},
        "gpu_launches": warm.kernel_launches * args.steps,
        "sub_batches": warm.sub_batches,
        "clocks": clk,
        "plain": {"value": plain, "unit": "volumes/s", "ms_per_volume": ms_plain / (args.steps * B),
                  "path": "n4_run, one volume per call, no warm start"},
        "batched_plain": {"value": world * B * args.steps / (ms_gplain / 1000.0), "unit": "volumes/s",
                          "ms_per_step": ms_gplain / args.steps, "path": "batch graph without warm start"},
        "warm_start": {"iterations_per_volume_warm": sum(iters_w) / B,
                       "iterations_per_volume_plain": sum(iters) / B, "kept": kept,
                       "max_abs_log_bias_diff_vs_plain_raw": max(draw),
                       "median_abs_log_bias_diff_vs_plain_raw": float(np.median(draw)),
                       "share_of_volumes_raw_within_0_01": float(np.mean(np.asarray(draw) <= 0.01)),
                       "max_abs_log_bias_diff_vs_plain_mean_removed": max(dcent),
                       "diff_basis": "per volume, max over the mask of |log bias (warm) - log bias (plain)| "
                                     "at full resolution; raw, and after removing its mean over the mask"},
        "autotune": {"cluster_sizes_ms": tune["candidates"], "chosen_cluster_size": tune["chosen"],
                     "chosen_threads": tune["chosen_threads"], "correction_tiles_ms": tune["correction"],
                     "chosen_correction_tile": tune["correction_chosen"], "sub_batches_ms": tune["sub_batches_ms"],
                     "chosen_sub_batches": tune["sub_batches_chosen"]},
        "batched_without_graph": {"value": world * B * args.steps / (ms_nograph / 1000.0), "unit": "volumes/s",
                                  "ms_per_step": ms_nograph / args.steps},
        "stages_ms_per_batch": dict(zip(("prologue", "n4_levels_iterations", "tables", "correction"), st_ms)),
        "stages_ms_per_batch_warm": dict(zip(("prologue_pool_encoder", "n4_levels_iterations", "tables",
                                              "correction"), t_w["stage_ms"])),
        "stage_gbs": {"correct": corr_gbs, "prologue": pro_gbs},
        "fit_gbs": comp["fit_gbs"],
        "upsample_gbs": comp["upsample_gbs"],
        "iterations_per_volume": sum(iters_w) / B,
        "c3_single_volume": c3,
        "c4_batched_uneven": c4,
        "host_enqueue_ms_per_step": host_ms,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_single()
    if rank == 0:
        print(json.dumps(line), flush=True)
    rep.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=96)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--components-only", action="store_true",
                    help="only the standalone fit / evaluation kernels at the 512x512x320 scale (for profiling)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", args.gpus))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        return run_reference(args, rank)
    if args.components_only:
        import torch
        import n4b200
        torch.cuda.set_device(local_rank)
        dev = torch.device("cuda", local_rank)
        print(json.dumps(measure_components(dev, n4b200.Context(local_rank), peaks()[0])), flush=True)
        return 0
    return run_ours(args, rank, world if "RANK" in os.environ else 1, local_rank)


if __name__ == "__main__":
    sys.exit(main())
