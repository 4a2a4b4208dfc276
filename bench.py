"""Benchmark of the batched tile correlator (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl b200|reference]

A step is one full correlation job: every tile pair of the workload (default
production_4096: 4096x4096 complex64 speckle pair, 14,400 pairs of 64x64 chips, +-32 px search,
refine factor 2 with an 8 px refine margin, zoom 8) run through the CUDA pipeline with rasters,
pair corners and outputs resident in HBM.  Under torchrun every rank correlates its own job of
the same size on its own GPU (weak scaling, no collective on the data path); ``value`` is the
pairs of all ranks divided by the slowest rank's device time.  With ``--shard`` the ranks split
one job into row bands instead, each holding only the raster lines its band reads (strong
scaling; ``value`` is the job's pairs over the slowest rank's time).

Beside the headline the line carries the reference's default tile geometry (128 x 128 chips,
32 px padding) as ``reference_default_geometry``, the serving loop over its whole range
(``serving``: latency with uploads, and a saturation run) and the uneven batch in one CUDA graph.

``e2e`` is the same metric through the host entry point of the C ABI
(ampcor_correlate_host): each step uploads both rasters and the corners from pinned host
memory, runs the job and reads the offsets back.

``--impl reference`` times the reference's own CPU implementation of the path instead: its
``Sequential`` correlator (lib/libampcor/correlators/Sequential.cc, the coarse correlation; its
refine() is empty), compiled unmodified into oracle/_ref/ against stand-ins of pyre, driven
through its own addReferenceTile / addTargetTile / adjust on tiles of the same rasters, one worker
per host thread, on a bounded sample of the same pairs each step.  Where oracle/_ref is not built
it times the FP64 restatement of the full pipeline in oracle/ instead (``kind: port``).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# nvidia-smi clock samples of the timed region (AMPCOR_CLOCK_DIR, else the system temp dir)
CLOCK_DIR = os.environ.get("AMPCOR_CLOCK_DIR") or tempfile.gettempdir()
METRIC = "tile pairs/s (64² chip, ±32 px search) & p99 job latency at ≤0.01 px error"
UNIT = "tile pairs/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="production_4096")
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--plain", action="store_true",
                    help="plain FP32 form only (no tensor-core candidates)")
    ap.add_argument("--no-tune", action="store_true",
                    help="skip the autotuner (default form and chunk)")
    ap.add_argument("--pairs", type=int, default=0,
                    help="correlate only the first N pairs (small cases for profiling)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-uneven", action="store_true")
    ap.add_argument("--shard", action="store_true",
                    help="with several ranks, split one job into row bands (strong scaling) "
                         "instead of running the job on every rank (weak scaling)")
    ap.add_argument("--no-geometries", action="store_true",
                    help="skip the chip-128 (reference default geometry) line")
    ap.add_argument("--serving-jobs", type=int, default=40)
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


def workload_config(w):
    return {
        "workload": (f"{w.name}: {w.ref.shape[0]}x{w.ref.shape[1]} complex64 raster pair, "
                     f"{w.pairs} pairs of {w.chip}x{w.chip} chips, +-{w.margin} px search, "
                     f"refine {w.refine_factor} (margin {w.refine_margin}), zoom {w.zoom_factor}"),
        "pairs_per_gpu": w.pairs,
        "chip": w.chip,
        "search_margin": w.margin,
        "refine_factor": w.refine_factor,
        "refine_margin": w.refine_margin,
        "zoom_factor": w.zoom_factor,
        "l2": "inputs larger than L2 (two 134 MB rasters per job; L2 is 126 MB)",
    }


def oracle_rate(w, seconds, threads):
    """Pairs/s of the FP64 CPU pipeline on a bounded sample of the workload's pairs."""
    import oracle

    rng = np.random.default_rng(0)
    order = rng.permutation(w.pairs)
    probe = order[: max(threads, 8)]
    t0 = time.perf_counter()
    oracle.adjust(w.ref, w.tgt, w.ulhc[probe], w.chip, w.window, w.refine_factor,
                  w.refine_margin, w.zoom_factor, threads=threads)
    per = (time.perf_counter() - t0) / len(probe)
    n = int(min(w.pairs, max(len(probe), seconds / max(per, 1e-9))))
    n = max(threads, (n // threads) * threads) if n >= threads else n
    sample = np.sort(order[:n])
    t0 = time.perf_counter()
    oracle.adjust(w.ref, w.tgt, w.ulhc[sample], w.chip, w.window, w.refine_factor,
                  w.refine_margin, w.zoom_factor, threads=threads)
    dt = time.perf_counter() - t0
    return n / dt, n, dt


def reference_rate(w, rasters, seconds, threads):
    """Pairs/s of the reference's own CPU correlator (oracle/_ref) on a bounded sample of the
    workload's pairs; ``rasters`` holds the raster files it reads (written before timing)."""
    from oracle import ref as refcpu

    rng = np.random.default_rng(0)
    order = rng.permutation(w.pairs)
    probe = np.sort(order[: max(threads, 8)])
    t0 = time.perf_counter()
    refcpu.sequential(rasters, w.ulhc[probe], w.chip, w.window, threads=threads)
    per = (time.perf_counter() - t0) / len(probe)
    n = int(min(w.pairs, max(len(probe), seconds / max(per, 1e-9))))
    n = max(threads, (n // threads) * threads) if n >= threads else n
    sample = np.sort(order[:n])
    t0 = time.perf_counter()
    refcpu.sequential(rasters, w.ulhc[sample], w.chip, w.window, threads=threads)
    dt = time.perf_counter() - t0
    return n / dt, n, dt


REFERENCE_SAMPLE = ("the reference's own CPU correlator (lib/libampcor/correlators/Sequential.cc "
                    "adjust(), FP64 coarse correlation, with its addReferenceTile/addTargetTile "
                    "reading the rasters as SLC files), compiled unmodified into oracle/_ref/ "
                    "against stand-ins of pyre, one worker per thread")


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(CLOCK_DIR, f"ampcor_clocks_rank{index}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
            time.sleep(0.6)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def fp32_peak(device):
    import ctypes

    path = os.path.join(ROOT, "ampcor_b200", "libampcor_peak.so")
    lib = ctypes.CDLL(path)
    lib.fp32_fma_tflops.restype = ctypes.c_double
    lib.fp32_fma_tflops.argtypes = [ctypes.c_int, ctypes.c_int]
    return lib.fp32_fma_tflops(device, 5)


SPEC_LENGTHS = (16, 24, 32, 40, 48, 64, 80, 96, 120, 128, 144, 160)


def spec_length(w):
    """The transform length the spectral form uses for a window of w samples."""
    return next((n for n in SPEC_LENGTHS if n >= w), 0)


def fft_flops(n):
    """Arithmetic of one complex n-point FFT, by the usual 5 n log2 n count."""
    return 5.0 * n * np.log2(n) if n > 1 else 0.0


def load_traffic():
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        return json.load(open(path))
    except Exception:
        return {}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import ref as refcpu
    from ampcor_b200 import synth

    w = synth.workload(args.workload)
    threads = os.cpu_count() or 1
    total_budget = 150.0
    per_step = max(2.0, total_budget / max(1, args.steps + args.warmup))
    rates, samples = [], []
    use_ref = refcpu.available()
    rasters = refcpu.Rasters(w.ref, w.tgt) if use_ref else None
    for i in range(args.warmup + args.steps):
        if use_ref:
            r, n, dt = reference_rate(w, rasters, per_step, threads)
        else:
            r, n, dt = oracle_rate(w, per_step, threads)
        if i >= args.warmup:
            rates.append(r)
            samples.append(n)
    if rasters:
        rasters.close()
    value = statistics.median(rates)
    what = (REFERENCE_SAMPLE if use_ref else
            "FP64 restatement of the full reference pipeline (oracle/oracle.c: coarse NCC, nudge, "
            "FFT refinement, refined NCC, zoom, offsets), OpenMP over pairs")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * w.pairs / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config(w),
        "cpu_baseline": {
            "value": value, "unit": UNIT, "cores": threads, "kind": "reference" if use_ref else "port",
            "sample": (f"{what}, on {threads} threads, {samples[0]} random pairs of the workload per "
                       f"step (median of {len(rates)} steps); ms_per_step is the whole job at that rate"),
        },
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_b200(args):
    import torch
    import torch.distributed as dist

    from ampcor_b200 import synth
    from ampcor_b200.worker import Worker

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)

    w = synth.workload(args.workload)
    if args.pairs:
        w.ulhc = w.ulhc[: args.pairs]
        w.truth = None if w.truth is None else w.truth[: args.pairs]
    # job pairs all ranks process per step: the job on every rank (weak scaling), or one job
    # split into row bands, each rank holding only the raster lines its band reads (strong)
    shard = args.shard and world > 1
    job_pairs = w.pairs * (1 if shard else world)
    if shard:
        import dataclasses

        from ampcor_b200 import parallel

        idx, ref_b, tgt_b, local = parallel.band(w.ref, w.tgt, w.ulhc, w.chip, w.window, rank, world)
        w = dataclasses.replace(w, ref=np.ascontiguousarray(ref_b), tgt=np.ascontiguousarray(tgt_b),
                                ulhc=local, centres=w.centres[idx],
                                truth=None if w.truth is None else w.truth[idx])
    worker = Worker(pairs=w.pairs, chip=(w.chip, w.chip), window=(w.window, w.window),
                    refine_factor=w.refine_factor, refine_margin=w.refine_margin,
                    zoom_factor=w.zoom_factor, device=local, plain=args.plain)
    ref = torch.from_numpy(w.ref).to(dev)
    tgt = torch.from_numpy(w.tgt).to(dev)
    ulhc = torch.from_numpy(w.ulhc).to(dev)
    offsets = torch.empty((w.pairs, 2), dtype=torch.float32, device=dev)

    tuned = None
    if not args.no_tune:
        from ampcor_b200.autotune import tune

        forms = ("plain",) if args.plain else ("spectral", "tensor", "plain")
        tuned = tune(worker, ref, tgt, ulhc, forms=forms, use_cache=False)

    def step():
        worker.correlate(ref, tgt, ulhc, offsets=offsets, synchronize=False)

    def barrier():
        if world > 1:
            dist.barrier()

    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    worker.profile(True)
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    kt = worker.kernel_times()
    launches = sum(n for _, n in kt.values())
    # timed regions per kernel kind: one per chunk of pairs and step (the plain form's coarse
    # kernel runs once per step over all pairs)
    nchunks = -(-w.pairs // max(int(worker.chunk), 1))
    kt_regions = {k: args.steps * nchunks for k in kt}
    if worker.form == "plain":
        kt_regions["coarse_correlation"] = args.steps
    worker.profile(False)
    clk = clocks.stop()
    # result check outside the timed region
    worker._lib.ampcor_synchronize(worker.handle, None)
    ok = bool(torch.isfinite(offsets).all().item())

    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = job_pairs * args.steps / (ms_max / 1000.0)

    # end to end through the host entry point, pinned host buffers
    e2e_value, e2e_steps = None, 0
    if not args.no_e2e:
        ref_h = torch.empty(w.ref.shape, dtype=torch.complex64, pin_memory=True)
        tgt_h = torch.empty(w.tgt.shape, dtype=torch.complex64, pin_memory=True)
        ulhc_h = torch.empty(w.ulhc.shape, dtype=torch.int32, pin_memory=True)
        ref_h.numpy()[...] = w.ref
        tgt_h.numpy()[...] = w.tgt
        ulhc_h.numpy()[...] = w.ulhc
        rn, tn, un = ref_h.numpy(), tgt_h.numpy(), ulhc_h.numpy()
        worker.correlate(rn, tn, un)
        e2e_steps = max(3, min(args.steps, 10))
        barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            out = worker.correlate(rn, tn, un)
        e2e_s = time.perf_counter() - t0
        te = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        e2e_value = job_pairs * e2e_steps / float(te.item())
        ok = ok and bool(np.isfinite(out).all())

    line = None
    if rank == 0:
        C = w.window - w.chip + 1
        E = w.chip + 2 * w.refine_margin
        Rf = w.refine_factor * w.chip
        Cf = 2 * w.refine_factor * w.refine_margin + 1
        f = w.refine_factor
        R, W, Wf = w.chip, w.window, f * E
        Z = w.zoom_factor * Cf
        # algorithmic work per pair of each kernel kind: the spectral kernels are bounded by the
        # bytes they must move (amplitude tiles in, placement statistics in, surfaces out), the
        # direct forms by the flops of the direct-form sums, the zoom by its two products
        if worker.form == "spectral":
            work = {
                "coarse_correlation": ("hbm", 4.0 * (W * W + R * R + C * C)),
                "refinement": ("hbm", 8.0 * (R * R + E * E) + 4.0 * (Rf * Rf + Wf * Wf)),
                "fine_correlation": ("hbm", 4.0 * (Wf * Wf + Rf * Rf + Cf * Cf)),
            }
        else:
            work = {
                "coarse_correlation": ("tensor", 2.0 * R ** 2 * C ** 2),
                "fine_correlation": ("tensor", 2.0 * Rf ** 2 * Cf ** 2),
                "refinement": ("tensor", 4.0 * (f * f - 1) * (R ** 3 + E ** 3)),
            }
        work["zoom"] = ("tensor", 2.0 * (Z * Cf * Cf + Z * Z * Cf))
        names = {
            "coarse_correlation": {"tensor": "tc_coarse_kernel", "spectral": "spec_staged_kernel (coarse)"}
            .get(worker.form, "coarse_kernel"),
            "fine_correlation": {"tensor": "tc_fine_kernel", "spectral": "spec_staged_kernel (fine)"}
            .get(worker.form, "fine_kernel"),
            "refinement": {"spectral": "spec_refine_kernel (chip + window)"}.get(worker.form, "refine_kernel"),
            "coarse_statistics": {"spectral": "detect_kernel + box_vsum_kernel + box_inv_kernel (per raster)"}
            .get(worker.form, "window_stats_cplx_kernel"),
            "fine_statistics": {"spectral": "spec_chip_stats_kernel + spec_tile_stats_kernel (blocked fine stage)"}
            .get(worker.form, "window_stats_real_kernel"),
            "zoom": "tc_zoom_kernel (zoom_kernel where Zm exceeds the tensor memory)",
        }
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except Exception:
            pass
        peak_src = "of measured" if peaks.get("bf16_tflops") else "of fallback"
        peak_of = {"hbm": (peaks.get("hbm_gbs") or 6650.0, "GB/s", 1e9),
                   "tensor": (peaks.get("bf16_tflops") or 1590.0, "TFLOP/s", 1e12)}
        simt = fp32_peak(local)
        traffic_table = load_traffic()
        kernels = {}
        for k, (bound, per_pair) in work.items():
            k_ms, k_n = kt.get(k, (0.0, 0))
            if not k_n or k_ms <= 0:
                continue
            regions = max(kt_regions.get(k, 1), 1)
            pairs_per_region = w.pairs * args.steps / regions
            amount = per_pair * pairs_per_region
            region_ms = k_ms / regions
            peak, unit, scale = peak_of[bound]
            if k == "zoom":
                peak = peak / 2.0  # tf32 runs at half the bf16 rate
            achieved = amount / (region_ms / 1000.0) / scale
            tr = traffic_table.get(names[k])
            kernels[k] = {"kernel": names[k], "bound": bound, "achieved": achieved, "peak": peak,
                          "unit": unit, "frac": achieved / peak, "ms_per_step": k_ms / args.steps,
                          "amount_per_region": amount, "ms_per_region": region_ms,
                          "traffic": tr["bytes_per_pair"] * pairs_per_region if tr else None}
        if worker.form == "spectral":
            # the spectral kernels are bound by instruction issue, not by memory: their FFT
            # arithmetic (5 N log2 N flops per complex N-point transform) against the measured FP32
            # FMA peak; a correlation runs W forward row transforms, N forward column transforms,
            # N / 2 + 1 inverse column transforms (the Hermitian half) and (C + 1) / 2 inverse row
            # transforms (two placement rows each)
            nc, nf = spec_length(W), spec_length(Wf)
            fft = {
                "coarse_correlation": (W + nc + nc // 2 + 1 + (C + 1) // 2) * fft_flops(nc),
                "fine_correlation": (Wf + nf + nf // 2 + 1 + (Cf + 1) // 2) * fft_flops(nf),
                "refinement": sum(n * fft_flops(n) + n * fft_flops(f * n) + f * n * fft_flops(n)
                                  + f * n * fft_flops(f * n) for n in (R, E)),
            }
            for k, per_pair in fft.items():
                if k in kernels:
                    kk = kernels[k]
                    t = per_pair * (kk["amount_per_region"] / work[k][1]) / (kk["ms_per_region"] / 1e3) / 1e12
                    kk["fft_flops_per_pair"] = per_pair
                    kk["fft_tflops"] = t
                    kk["fft_frac_of_fp32_simt"] = t / simt
        top = max(kernels, key=lambda k: kernels[k]["ms_per_step"])
        topk = kernels[top]
        cpu = None
        parity_rep = None
        if world == 1 and not args.no_cpu_baseline:
            cpu, parity_rep = cpu_leg(w, worker, ref, tgt, ulhc, offsets)
        h2d = w.ref.nbytes + w.tgt.nbytes + w.ulhc.nbytes
        d2h = w.pairs * 2 * 4
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "strong" if shard else "weak", "vs_baseline": None,
            "dtype": "bf16x3" if worker.form == "tensor" else "f32",
            "data": "synthetic",
            "config": dict(workload_config(w), form=worker.form, chunk=worker.chunk,
                           autotuned=tuned is not None,
                           tune=[(c["form"], c["chunk"], round(c["ms"], 3)) for c in tuned["candidates"]]
                           if tuned else None),
            "roofline": {
                "bound": topk["bound"], "kernel": topk["kernel"], "achieved": topk["achieved"],
                "peak": topk["peak"], "unit": topk["unit"], "frac": topk["frac"],
                "traffic": topk["traffic"],
                "peak_note": (f"{'HBM copy bandwidth' if topk['bound'] == 'hbm' else 'dense bf16 tensor throughput'} "
                              f"{peak_src} (MEASURED_PEAKS.json); achieved = algorithmic "
                              f"{'bytes' if topk['bound'] == 'hbm' else 'flops'} of one timed region "
                              f"(one chunk of pairs) / its CUDA-event time; traffic from "
                              f"profiles/traffic.json (ncu)"),
                "fp32_simt_peak": simt,
                "top_kernel_fft_frac_of_fp32_simt": topk.get("fft_frac_of_fp32_simt"),
                "kernels": kernels,
                "kernel_ms_per_step": {names[k]: v[0] / args.steps for k, v in kt.items() if v[1]},
                "launches_per_step": {names[k]: v[1] / args.steps for k, v in kt.items() if v[1]},
            },
            "e2e": ({"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                     "d2h_bytes_per_step": d2h, "steps": e2e_steps} if e2e_value else None),
            "gpu_launches": int(launches + args.steps),  # + the corner-offset kernel per step
            "clocks": clk,
            "results_finite": ok,
        }
        if cpu:
            line["cpu_baseline"] = cpu
        if parity_rep:
            line["parity"] = parity_rep
        if world == 1 and not args.no_geometries:
            line["reference_default_geometry"] = geometry_run("reference_default_4096", local, args)
        if world == 1 and not args.no_serving:
            line["serving"] = serving_run(local, args)
        if world == 1 and not args.no_uneven:
            line["batched_uneven"] = uneven_run(local, args)
        print(json.dumps(line), flush=True)
    worker.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def cpu_leg(w, worker, ref, tgt, ulhc, timed_offsets):
    """The CPU baseline and the parity check of the timed job, outside the timed region.  The
    baseline is the reference's own CPU correlator (oracle/_ref) on a bounded sample of the job's
    pairs, on all host threads (the FP64 oracle's whole-job time where oracle/_ref is not built).
    The FP64 oracle runs the whole job once, and the timed job's offsets are checked against it
    pair by pair (oracle.parity.compare; the same worker reruns the job with diagnostics and
    surfaces, and its offsets must equal the timed ones bit for bit)."""
    import torch

    from oracle import parity
    from ampcor_b200.worker import DIAG_DTYPE

    from oracle import ref as refcpu

    dev = ref.device
    P = w.pairs
    diag = torch.zeros((P, DIAG_DTYPE.itemsize), dtype=torch.uint8, device=dev)
    cs = torch.zeros((P, worker.coarse_dim, worker.coarse_dim), dtype=torch.float32, device=dev)
    rs = torch.zeros((P, worker.refined_dim, worker.refined_dim), dtype=torch.float32, device=dev)
    off = worker.correlate(ref, tgt, ulhc, diag=diag, coarse_surfaces=cs, refined_surfaces=rs)
    same_as_timed = bool(torch.equal(off, timed_offsets))
    gpu_off = timed_offsets.cpu().numpy()
    gpu_diag = diag.cpu().numpy().view(DIAG_DTYPE).reshape(P)
    cs_h, rs_h = cs.cpu().numpy(), rs.cpu().numpy()
    del cs, rs
    threads = os.cpu_count() or 1
    orc = parity.oracle_run(w.ref, w.tgt, w.ulhc, w.chip, w.window, w.refine_factor,
                            w.refine_margin, w.zoom_factor, threads=threads)
    dt = orc["adjust_seconds"]
    if refcpu.available():
        with refcpu.Rasters(w.ref, w.tgt) as rasters:
            rate, n, rdt = reference_rate(w, rasters, 15.0, threads)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
               "sample": f"{REFERENCE_SAMPLE}: {n} random pairs of the workload, {rdt:.1f} s on {threads} threads"}
    else:
        cpu = {"value": P / dt, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": (f"the whole job ({P} pairs) through the FP64 restatement of the full "
                          f"reference pipeline (oracle/oracle.c: coarse NCC, nudge, FFT refinement, "
                          f"refined NCC, zoom, offsets), OpenMP over pairs, {dt:.1f} s on {threads} "
                          f"threads")}
    rep = parity.summary(parity.compare(orc, gpu_off, gpu_diag, cs_h, rs_h))
    rep["oracle_pairs_per_s"] = P / dt
    rep["rerun_equals_timed_offsets"] = same_as_timed
    rep["rule"] = ("every pair against the FP64 oracle: cells equal (offsets then bit-exact) "
                   "unless the pair's own measured surface error explains a near-tie, counted "
                   "in pairs_excused; oracle/parity.py")
    return cpu, rep


def serving_run(device, args):
    """The continuous-batching loop over the serving range (square rasters of 1024^2 to 8192^2,
    chips 32-128, margins 16-64, refine 2, zoom 8-16): p50 / p99 job latency under a seeded Poisson
    stream of 20 jobs/s with each job's upload from pinned host memory inside its latency, then the
    same jobs queued all at once with their rasters in device memory (the rate the loop sustains
    when work waits)."""
    import dataclasses

    import torch

    from ampcor_b200 import serve

    jobs = serve.poisson_jobs(args.serving_jobs, rate=20.0, seed=7, device=f"cuda:{device}",
                              sizes=(1024, 2048, 4096, 8192), chips=(32, 64, 128),
                              margins=(16, 32, 64), zooms=(8, 16), spacing=(64, 128), pinned=True,
                              square=True)
    srv = serve.Server(device=device, slots=3)
    srv.warm(jobs)
    srv.run(jobs, realtime=True)
    rep = serve.latency_report(jobs)
    dev = torch.device("cuda", device)
    queued = [dataclasses.replace(j, arrival=0.0, ref=j.ref.to(dev), tgt=j.tgt.to(dev), start=None,
                                  done=None, offsets=None) for j in jobs]
    torch.cuda.synchronize(dev)
    srv.run(queued, realtime=False)
    sat = serve.latency_report(queued)
    rep["saturation_pairs_per_s"] = sat["pairs_per_s"]
    rep["saturation_span_ms"] = 1e3 * max(j.done for j in queued)
    rep["saturation_same_offsets"] = all(np.array_equal(a.offsets, b.offsets) for a, b in zip(jobs, queued))
    rep["geometries"] = len({j.geometry for j in jobs})
    # the loop at the headline geometry (64 x 64 chips, +-32 px, zoom 8): 24 jobs on rasters of
    # 1024^2 to 8192^2 queued at once, against the 1.41M pairs/s of one whole job
    prod = serve.poisson_jobs(24, rate=20.0, seed=8, device=f"cuda:{device}",
                              sizes=(1024, 2048, 4096, 8192), chips=(64,), margins=(32,), zooms=(8,),
                              spacing=(33, 64), pinned=False, square=True)
    for j in prod:
        j.arrival = 0.0
    psrv = serve.Server(device=device, slots=3)
    psrv.warm(prod)
    psrv.run(prod, realtime=False)
    prep = serve.latency_report(prod)
    rep["saturation_headline_geometry_pairs_per_s"] = prep["pairs_per_s"]
    rep["saturation_headline_geometry_pairs"] = prep["pairs"]
    rep["stream"] = (f"{args.serving_jobs} jobs, Poisson 20 jobs/s (seed 7), square rasters of 1024, "
                     f"2048, 4096 or 8192 px (upload from pinned host memory inside each job's "
                     f"latency), chip 32/64/128, margin 16/32/64, refine 2, zoom 8/16, 3 slots; "
                     f"saturation: the same jobs queued at once, rasters in device memory; "
                     f"headline-geometry saturation: 24 jobs of 64 x 64 chips, +-32 px, zoom 8, "
                     f"rasters 1024^2-8192^2, queued at once")
    return rep


def geometry_run(name, device, args):
    """Throughput of another tile geometry beside the headline: workload ``name`` autotuned,
    warm-up and timed jobs with everything device-resident (CUDA events), then end to end through
    ampcor_correlate_host with pinned host rasters."""
    import torch

    from ampcor_b200 import synth
    from ampcor_b200.autotune import tune
    from ampcor_b200.worker import Worker

    w = synth.workload(name)
    dev = torch.device("cuda", device)
    worker = Worker(pairs=w.pairs, chip=(w.chip, w.chip), window=(w.window, w.window),
                    refine_factor=w.refine_factor, refine_margin=w.refine_margin,
                    zoom_factor=w.zoom_factor, device=device)
    ref = torch.from_numpy(w.ref).to(dev)
    tgt = torch.from_numpy(w.tgt).to(dev)
    ulhc = torch.from_numpy(w.ulhc).to(dev)
    offsets = torch.empty((w.pairs, 2), dtype=torch.float32, device=dev)
    tuned = tune(worker, ref, tgt, ulhc, forms=("spectral", "tensor", "plain"), use_cache=False)
    for _ in range(max(args.warmup, 3)):
        worker.correlate(ref, tgt, ulhc, offsets=offsets, synchronize=False)
    steps = max(3, min(args.steps, 10))
    torch.cuda.synchronize()
    worker.profile(True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        worker.correlate(ref, tgt, ulhc, offsets=offsets, synchronize=False)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    kt = worker.kernel_times()
    worker.profile(False)
    worker._lib.ampcor_synchronize(worker.handle, None)
    ref_h = torch.empty(w.ref.shape, dtype=torch.complex64, pin_memory=True)
    tgt_h = torch.empty(w.tgt.shape, dtype=torch.complex64, pin_memory=True)
    ref_h.numpy()[...] = w.ref
    tgt_h.numpy()[...] = w.tgt
    un = np.ascontiguousarray(w.ulhc)
    worker.correlate(ref_h.numpy(), tgt_h.numpy(), un)
    t0 = time.perf_counter()
    for _ in range(3):
        out = worker.correlate(ref_h.numpy(), tgt_h.numpy(), un)
    e2e_s = (time.perf_counter() - t0) / 3
    line = {
        "workload": workload_config(w)["workload"], "pairs": w.pairs, "form": worker.form,
        "chunk": worker.chunk, "steps": steps, "ms_per_job": ms, "pairs_per_s": w.pairs / (ms / 1e3),
        "e2e_pairs_per_s": w.pairs / e2e_s,
        "kernel_ms_per_job": {k: v[0] / steps for k, v in kt.items() if v[1]},
        "tune": [(c["form"], c["chunk"], round(c["ms"], 3)) for c in tuned["candidates"]],
        "results_finite": bool(np.isfinite(out).all()),
    }
    worker.close()
    return line


def uneven_run(device, args):
    """Throughput of the batched uneven configuration: 16 raster pairs of different sizes and
    geometries, every geometry autotuned, all work replayed as one CUDA graph."""
    import torch

    from ampcor_b200 import batch

    jobs = batch.uneven_jobs(16, seed=11, device=f"cuda:{device}")
    ub = batch.UnevenBatch(jobs, device=device, tune=True)
    ub.capture()
    for _ in range(2):
        ub.replay()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    reps = 5
    with torch.cuda.stream(ub.stream):
        e0.record()
        for _ in range(reps):
            ub.replay()
        e1.record()
    torch.cuda.synchronize()
    ub.check()
    ms = e0.elapsed_time(e1) / reps
    geoms = sorted({j.geometry for j in jobs})
    out = {
        "raster_pairs": len(jobs), "pairs": ub.pairs, "ms_per_batch": ms,
        "pairs_per_s": ub.pairs / (ms / 1e3),
        "geometries": [f"chip {g[0]} margin {g[1]} zoom {g[4]}: "
                       f"{ub.tuning[g]['form']} chunk {ub.tuning[g]['chunk']}" for g in geoms],
        "launch": "one CUDA graph replay per batch",
    }
    ub.close()
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
