"""Benchmark: photons/s of the propagation hot path on the light-field
telescope scene (the refraction-heavy configuration: a 252-facet f=10.7 m
Davies-Cotton reflector with a light-field sensor of 1039 bi-convex lenses
and 63,379 hexagonal lixels in its focal plane).

One step = propagate one batch of photons (supports uniform on a 5.55 m
disc 21.4 m above the dish, directions within 1.5 degrees of -z, wavelength
300-700 nm, max. 10 interactions) and bin the arrivals per lixel.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
                    [--tracer fp64|fp32] [--photons P]

For N > 1 it runs under torch.distributed.run, one process per GPU; every
rank traces its own batch (weak scaling) and the step time is the maximum
over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

SCENE = dict(focal_length=10.7, aperture_radius=5.35, fov_deg=6.5, pixel_fov_deg=0.186,
             paxels_on_diagonal=9, housing_overhead=1.1, reflectivity=0.9)
SOURCE = dict(disc_radius=5.55, height=21.4, max_zenith_deg=1.5)
MAX_INTERACTIONS = 10
# algorithmic HBM bytes per photon: in 7 x f64 + id (60 B), out sensor id,
# x, y, time (28 B); FP32 form: in 7 x f32 + id (32 B), out id + x, y f32 +
# time f64 (20 B)
BYTES_PER_PHOTON = {"fp64": 88, "fp64_plain": 88, "fp32": 52}
# FLOP weights of the operation counts (nodes tested, leaves transformed,
# cap quadratics, cap bounds, plane tests, other quadrics, reflections,
# Fresnel steps, time-of-flight segments, table look-ups)
FLOP_WEIGHTS = {"nodes": 26, "leaves": 48, "caps": 29, "cap_bounds": 85, "planes": 36,
                "others": 29, "reflections": 91, "fresnels": 110, "segments": 3, "funcs": 4}
# the kernel class that does each counted operation
FLOP_STAGE = {"nodes": "walk", "leaves": "intersect", "caps": "intersect",
              "cap_bounds": "intersect", "planes": "intersect", "others": "intersect",
              "reflections": "resolve", "fresnels": "resolve", "segments": "resolve",
              "funcs": "resolve"}
FP64_PEAK_TFLOPS_NOMINAL = 37.0   # B200 vector FP64 with FMAs, nominal
# DRAM bytes per photon of each kernel class on the light-field telescope,
# from an ncu capture of the timed step of 4e6 photons (dram__bytes_read.sum
# + dram__bytes_write.sum summed over the class's launches, divided by the
# photons of the step; profiles/wavefront_fp64_light_field_telescope.md):
# walk = the BVH level kernels; intake = intake + counter kernel;
# intersect = intersection + tie kernels; resolve = overflow walk +
# resolve + counter kernel; bin = zeroing + binning kernels.  The tracing
# order's kernels (run once per call, before the first iteration) are in
# no class (ORDER_DRAM_BYTES_PER_PHOTON).  The traffic of a step grows with its photons
# (the same scene and pool), so the bench scales these figures by its own
# photon count.
STAGE_DRAM_BYTES_PER_PHOTON = {"walk": 807.0, "intake": 247.5, "intersect": 1079.9,
                               "resolve": 897.4, "bin": 4.0}
ORDER_DRAM_BYTES_PER_PHOTON = 188.0
FP32_PEAK_TFLOPS_NOMINAL = 75.0   # B200 vector FP32 (non-tensor), nominal
WORKLOAD = "light-field telescope, 1039 lenses x 61 lixels (config 1)"
# the signal chain after binning (workload "signal"): quantum efficiency,
# dark rate [1/s], crosstalk, night-sky background flux [1/(s sr m^2 m)],
# exposure, time slice and single-photon time resolution [s]
SIGNAL = dict(qe=[[200e-9, 0.0], [450e-9, 0.6], [1200e-9, 0.0]], dark_rate=5e6, crosstalk=0.1,
              nsb_flux=[[250e-9, 1e17], [400e-9, 3e17], [700e-9, 2e17]], exposure=50e-9,
              time_slice=0.5e-9, time_std=0.4e-9)


def scene_config_name():
    return (f"f{SCENE['focal_length']}m_R{SCENE['aperture_radius']}m_fov{SCENE['fov_deg']}deg_"
            f"pix{SCENE['pixel_fov_deg']}deg")


def make_photons(n: int, seed: int):
    from merlict_development_kit_b200 import photons as P
    return P.downward_disc_source(n, seed, SOURCE["disc_radius"], SOURCE["height"],
                                  SOURCE["max_zenith_deg"])


def load_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def flop_counts():
    p = os.path.join(REPO, "tests", "golden", "flop_counts.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f)


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def init_dist():
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and not dist.is_initialized():
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        from datetime import timedelta
        dist.init_process_group(backend=backend, timeout=timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if torch.cuda.is_available() and dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---- reference arm ------------------------------------------------------------

def cpu_reference_run(photons_per_step: int, steps: int, warmup: int, threads_mode: str = "multi"):
    """The reference's own multi-threaded CPU path (merlict_multi_thread) plus
    Sensors::assign_photons, on the same scene built by the reference's own
    factories; returns (photons/s, seconds, cores, kind, sample)."""
    from oracle import oracle as O
    if O.harness_available():
        scene = O.RefScene("light_field_sensor",
                           (SCENE["focal_length"], SCENE["aperture_radius"], SCENE["fov_deg"],
                            SCENE["pixel_fov_deg"], SCENE["paxels_on_diagonal"],
                            SCENE["housing_overhead"], SCENE["reflectivity"]))
        mode = O.REFERENCE_MULTI_THREAD if threads_mode == "multi" else O.REFERENCE_SINGLE_THREAD
        cores = scene.lib.ref_hardware_concurrency() if threads_mode == "multi" else 1
        secs = []
        for k in range(warmup + steps):
            ph = make_photons(photons_per_step, 1000 + k)
            _, _, sec = scene.propagate(ph, MAX_INTERACTIONS, mode, seed=1 + k, results=False)
            if k >= warmup:
                secs.append(sec)
        total = float(sum(secs))
        what = ("merlict_multi_thread" if threads_mode == "multi"
                else "propagate_photons_in_frame_with_config (one thread)")
        return photons_per_step * steps / total, total, cores, "reference", \
            f"{steps} x {photons_per_step} photons, reference {what} + assign_photons"
    # the C restatement when the reference library is not built here
    from merlict_development_kit_b200 import factories as F
    flat = F.light_field_telescope(**SCENE).flatten()
    o = O.Oracle()
    secs = []
    for k in range(warmup + steps):
        ph = make_photons(photons_per_step, 1000 + k)
        t0 = time.perf_counter()
        o.propagate(flat, ph, MAX_INTERACTIONS, seed=1 + k)
        if k >= warmup:
            secs.append(time.perf_counter() - t0)
    total = float(sum(secs))
    return photons_per_step * steps / total, total, 1, "port", \
        f"{steps} x {photons_per_step} photons, C restatement, 1 thread"


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    per_step = args.ref_photons
    value, secs, cores, kind, sample = cpu_reference_run(per_step, args.steps, args.warmup)
    line = {
        "metric": "photons/s", "value": value, "unit": "photons/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": WORKLOAD, "scene": scene_config_name(),
                   "photons_per_step": per_step, "max_interactions": MAX_INTERACTIONS},
        "cpu_baseline": {"value": value, "unit": "photons/s", "cores": cores, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "photons/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---- our arm ------------------------------------------------------------------

def run_ours(args, world, rank, local):
    import torch
    from merlict_development_kit_b200 import engine, factories as F, _native
    import ctypes as C
    from merlict_development_kit_b200 import abi

    torch.cuda.set_device(local)
    flat = F.light_field_telescope(**SCENE).flatten()
    scene = engine.Scene(flat)
    n = args.photons
    tracer = args.tracer
    in_dtype = torch.float32 if tracer == "fp32" else torch.float64
    host = make_photons(n, 12345 + rank)
    dev = engine.photons_to_device(host, dtype=in_dtype)
    out_dtype = torch.float32 if tracer == "fp32" else torch.float64
    cfg = engine.PropagationConfig(MAX_INTERACTIONS)
    rng = engine.Philox(seed=7 + rank)
    stream = torch.cuda.current_stream()
    results = {}

    tuning = None
    if args.autotune and tracer != "fp64_plain":
        sample = {k: v[:min(n, 2_000_000)].contiguous() for k, v in dev.items()}
        tuning, _ = scene.autotune(sample, cfg, engine.Philox(3), tracer=tracer)
        del sample

    def step(ev=None):
        if ev is not None:
            ev[0].record(stream)
        out = scene.propagate(dev, cfg, rng, tracer=tracer, outputs=("sensor", "x", "y", "time"),
                              out_dtype=out_dtype, sync=False, results=results, tuning=tuning)
        if ev is not None:
            ev[1].record(stream)
        scene.bin_arrivals(out["sensor"])
        return out

    for _ in range(args.warmup):
        step()
    scene.sync_errors()
    torch.cuda.synchronize()

    kernel_events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                     for _ in range(args.steps)]
    clocks = ClockSampler(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    t_start = torch.cuda.Event(enable_timing=True)
    t_stop = torch.cuda.Event(enable_timing=True)
    launches0 = scene.kernel_launches()
    # the timed steps as one NVTX range, so that a profiler can capture
    # exactly their launches (ncu --nvtx --nvtx-include "bench_timed/")
    torch.cuda.nvtx.range_push("bench_timed")
    t_start.record(stream)
    for k in range(args.steps):
        step(kernel_events[k])
    t_stop.record(stream)
    torch.cuda.nvtx.range_pop()
    launches = scene.kernel_launches() - launches0
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    scene.sync_errors()
    # per-stage device times: the same steps again with CUDA events around
    # every kernel class (launched one by one, outside the timed region)
    scene.set_profiling(True)
    for k in range(args.steps):
        step()
    torch.cuda.synchronize()
    stage = scene.kernel_times()
    scene.set_profiling(False)
    elapsed_ms = t_start.elapsed_time(t_stop)
    kernel_ms = float(np.mean([a.elapsed_time(b) for a, b in kernel_events]))
    elapsed_ms = max_over_ranks(elapsed_ms, world)
    value = n * world * args.steps / (elapsed_ms * 1e-3)

    # the FP32 form on the same photons (rounded to FP32) with the same
    # Philox streams as one FP64 step: photons/s, replay-mode sensor
    # agreement and the per-lixel histogram divergence against FP64
    forms = None
    if tracer == "fp64" and not args.no_forms:
        from merlict_development_kit_b200.precision import js_divergence
        dev32 = {k: v.float() for k, v in dev.items()}
        dev64r = {k: v.double() for k, v in dev32.items()}
        tune32, _ = (scene.autotune({k: v[:min(n, 2_000_000)].contiguous() for k, v in dev32.items()},
                                    cfg, engine.Philox(3), tracer="fp32")
                     if args.autotune else (None, 0.0))
        ref = scene.propagate(dev64r, cfg, engine.Philox(31), outputs=("sensor",), tuning=tuning)
        ref_sensor = ref["sensor"].clone()
        res32 = {}
        for _ in range(2):
            scene.propagate(dev32, cfg, engine.Philox(31), tracer="fp32", outputs=("sensor",),
                            out_dtype=torch.float32, results=res32, tuning=tune32, sync=False)
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            scene.propagate(dev32, cfg, engine.Philox(31), tracer="fp32", outputs=("sensor",),
                            out_dtype=torch.float32, results=res32, tuning=tune32, sync=False)
        f1.record(stream)
        torch.cuda.synchronize()
        ms32 = max_over_ranks(f0.elapsed_time(f1) / args.steps, world)
        s32 = res32["sensor"]

        def hist(sn):
            sn = sn[sn >= 0].long()
            return torch.bincount(sn, minlength=flat.num_sensors).double().cpu().numpy()
        forms = {"fp32": {"value": n * world / (ms32 * 1e-3), "unit": "photons/s",
                          "replay_sensor_agreement": float((s32 == ref_sensor).float().mean()),
                          "lixel_js_vs_fp64": js_divergence(hist(s32), hist(ref_sensor)),
                          "tuning": tune32}}
        del dev32, dev64r, ref, res32

    # e2e: the C-ABI host-buffer call that does a step's whole work --
    # H2D of the batch, trace, per-lixel binning, D2H of the per-photon
    # results and the lixel counts, synchronise -- pinned host memory, same
    # batch size (mlgpu_propagate_and_bin_host: merlict's propagate +
    # Sensors::assign_photons pair)
    pin = {k: torch.from_numpy(np.ascontiguousarray(host[k])).to(in_dtype).pin_memory()
           for k in ("support_x", "support_y", "support_z", "direction_x", "direction_y",
                     "direction_z", "wavelength")}
    ph = abi.mlgpu_photons()
    ph.dtype = abi.F64 if in_dtype == torch.float64 else abi.F32
    for k, t in pin.items():
        setattr(ph, k, t.data_ptr())
    h_sensor = torch.empty(n, dtype=torch.int32).pin_memory()
    h_x = torch.empty(n, dtype=out_dtype).pin_memory()
    h_y = torch.empty(n, dtype=out_dtype).pin_memory()
    h_t = torch.empty(n, dtype=torch.float64).pin_memory()
    h_counts = torch.empty(flat.num_sensors, dtype=torch.int32).pin_memory()
    res = abi.mlgpu_results()
    res.dtype = abi.F64 if out_dtype == torch.float64 else abi.F32
    res.sensor, res.x, res.y, res.time = (h_sensor.data_ptr(), h_x.data_ptr(), h_y.data_ptr(),
                                          h_t.data_ptr())
    st = engine._settings(cfg, 0, tracer, "bvh", tuning)
    r = abi.mlgpu_rng()
    r.mode = abi.RNG_PHILOX
    r.seed = 99 + rank
    L = _native.lib()
    e2e_steps = max(1, min(args.steps, 5))

    def host_step():
        _native.check(L.mlgpu_propagate_and_bin_host(
            scene.handle, C.byref(ph), n, C.byref(st), C.byref(r), C.byref(res),
            C.c_void_p(h_counts.data_ptr()), None, 0, 0.0, 0.0))
    for _ in range(1):
        host_step()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        host_step()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    e2e_value = n * world * e2e_steps / e2e_s
    elt = 8 if in_dtype == torch.float64 else 4
    eout = 8 if out_dtype == torch.float64 else 4
    h2d = 7 * elt * n
    d2h = (4 + 2 * eout + 8) * n + 4 * flat.num_sensors
    del pin, h_sensor, h_x, h_y, h_t, dev
    torch.cuda.empty_cache()
    # the other configurations' forms, each on its own scene and photons
    if tracer == "fp64" and not args.no_forms:
        clk_forms = ClockSampler(local)
        clk_forms.start()
        forms = forms or {}
        forms["batched_events"] = bunches_form(flat, args.events, 2, 1, world, rank, local)
        forms["precision"] = precision_form(args.precision_photons, 2, 1, world, rank, local)
        forms["clocks"] = clk_forms.stop()

    if rank != 0:
        return
    hbm_peak, peak_kind = load_peaks()
    bpp = BYTES_PER_PHOTON[tracer]
    fp32 = tracer == "fp32"
    vec_peak = FP32_PEAK_TFLOPS_NOMINAL if fp32 else FP64_PEAK_TFLOPS_NOMINAL
    counts = flop_counts()
    per = counts["per_photon"] if counts else {}
    stage_flops = {}
    for k, w in FLOP_WEIGHTS.items():
        stage_flops[FLOP_STAGE[k]] = stage_flops.get(FLOP_STAGE[k], 0.0) + w * per.get(k, 0.0)
    total_stage_ms = sum(ms for ms, _ in stage.values())
    kernels = {}
    for name, (ms, nl) in stage.items():
        if nl == 0:
            continue
        f = stage_flops.get(name, 0.0) * n * args.steps
        kernels[name] = {"ms_per_step": ms / args.steps, "launches": nl,
                         "avg_launch_ms": ms / nl, "share": ms / total_stage_ms,
                         "flops_per_photon": stage_flops.get(name, 0.0),
                         "tflops": f / (ms * 1e-3) / 1e12 if ms > 0 else None}
    dominant = max(kernels, key=lambda k: kernels[k]["ms_per_step"])
    dk = kernels[dominant]
    # the dominant stage against the vector pipe that bounds it: the
    # reference's operation counts for that stage, per photon, times the
    # photons of a step, over the stage's device time per step
    achieved = dk["flops_per_photon"] * n / (dk["ms_per_step"] * 1e-3) / 1e12
    # the denominator, measured on this GPU: separate FP64 adds and
    # multiplies (the reference's operations, which the bit-exact tracer may
    # not contract into FMAs), with the FMA rate beside it
    rate_addmul, rate_fma = C.c_double(0.0), C.c_double(0.0)
    _native.check(L.mlgpu_probe_fp64_rate(0, C.byref(rate_addmul), None))
    _native.check(L.mlgpu_probe_fp64_rate(1, C.byref(rate_fma), None))
    peak = rate_addmul.value / 1e12 if not fp32 else vec_peak
    traffic = STAGE_DRAM_BYTES_PER_PHOTON.get(dominant)
    roofline = {"bound": "fp32" if fp32 else "fp64", "kernel": dominant,
                "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak,
                "traffic": traffic * n / dk["launches"] * args.steps if traffic else None,
                "traffic_unit": "DRAM bytes per launch of the stage (ncu, scaled by photons)",
                "peak_source": ("measured on this GPU: FP64 adds and multiplies "
                                "(mlgpu_probe_fp64_rate, no FMA)" if not fp32 else
                                "nominal B200 vector FP32 peak (no measured figure)"),
                "peak_fp64_fma_measured": rate_fma.value / 1e12,
                "frac_of_fma_peak": achieved / (rate_fma.value / 1e12),
                "peak_fp64_nominal": FP64_PEAK_TFLOPS_NOMINAL,
                "flops_per_photon": dk["flops_per_photon"]}
    flops = sum(stage_flops.values())
    whole = flops * n / (kernel_ms * 1e-3) / 1e12
    compute = {"bound": roofline["bound"], "flops_per_photon": flops, "achieved": whole,
               "peak": peak, "unit": "TFLOP/s", "frac": whole / peak,
               "scope": "whole propagate call"}
    achieved_gbs = bpp * n / (kernel_ms * 1e-3) / 1e9
    hbm = {"bound": "hbm", "achieved": achieved_gbs, "peak": hbm_peak, "unit": "GB/s",
           "frac": achieved_gbs / hbm_peak,
           "peak_source": ("measured: MEASURED_PEAKS.json hbm_gbs" if peak_kind == "measured"
                           else "fallback: 6,650 GB/s of the profiling recipe (no "
                                "MEASURED_PEAKS.json)"),
           "bytes_per_photon": bpp, "scope": "whole propagate call"}
    if STAGE_DRAM_BYTES_PER_PHOTON and not fp32:
        # the FP64 tracer's measured DRAM traffic (ncu, all kernel classes and
        # the tracing order) against the algorithmic bytes
        measured = sum(STAGE_DRAM_BYTES_PER_PHOTON.values()) + ORDER_DRAM_BYTES_PER_PHOTON
        hbm["dram_bytes_per_photon_measured"] = measured
        hbm["dram_over_algorithmic"] = measured / bpp
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        v, secs, cores, kind, sample = cpu_reference_run(args.ref_photons, 2, 1)
        cpu = {"value": v, "unit": "photons/s", "cores": cores, "kind": kind, "sample": sample}
        # merlict's single-thread loop (Photons.cpp:9-22), which beats its
        # thread pool on cheap scenes
        v1, _, c1, k1, s1 = cpu_reference_run(args.ref_photons // 5, 2, 1, threads_mode="single")
        cpu["single_thread"] = {"value": v1, "unit": "photons/s", "cores": c1, "kind": k1,
                                "sample": s1}
    line = {
        "metric": "photons/s", "value": value, "unit": "photons/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if fp32 else "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "scene": scene_config_name(), "tracer": tracer,
                   "photons_per_step_per_gpu": n, "max_interactions": MAX_INTERACTIONS,
                   "l2": "inputs larger than L2 (photon planes %.0f MB)" % (7 * elt * n / 1e6),
                   "tuning": tuning or "defaults",
                   "stage_times": "a second pass over the same steps, kernels timed one by one"},
        "kernel_ms": kernel_ms,
        "roofline": roofline,
        "compute_roofline": compute,
        "hbm_roofline": hbm,
        "kernels": kernels,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "photons/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "forms": forms,
        "gpu_launches": launches,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    scene.close()


def bunches_form(flat, events: int, steps: int, warmup: int, world: int, rank: int, local: int,
                 seed: int = 0):
    """Batched uneven events (config 2): `events` air-shower-like events with
    log-uniform sizes in [1e2, 1e6] photons on the light-field telescope,
    traced (a) as one photon stream with autotuned knobs and CUDA-graph
    launches and (b) with one propagate call per event (the reference's
    per-event loop, plenoscope_propagation.cpp:206-210), same Philox streams,
    so the two give identical results.  Returns the form's line items."""
    import torch
    from merlict_development_kit_b200 import engine, photons as P

    scene = engine.Scene(flat)
    sizes = P.cherenkov_event_sizes(events, 2024 + rank + seed)
    dev, off = P.cherenkov_events(sizes, 4048 + rank + seed, device=f"cuda:{local}")
    n = int(off[-1])
    cfg = engine.PropagationConfig(MAX_INTERACTIONS)
    stream = torch.cuda.current_stream()
    outs = ("sensor", "x", "y", "time")
    sample = {k: v[:min(n, 4_000_000)].contiguous() for k, v in dev.items()}
    tuning, _ = scene.autotune(sample, cfg, engine.Philox(3))
    del sample
    res_batched, res_events = {}, {}

    def batched():
        return scene.propagate(dev, cfg, engine.Philox(11), outputs=outs, sync=False,
                               results=res_batched, tuning=tuning)

    def per_event():
        for e in range(len(sizes)):
            a, b = int(off[e]), int(off[e + 1])
            part = {k: v[a:b] for k, v in dev.items()}
            r = {k: v[a:b] for k, v in res_events.items()}
            scene.propagate(part, cfg, engine.Philox(11, photon_offset=a), outputs=outs,
                            sync=False, results=r)

    for _ in range(warmup):
        batched()
    scene.sync_errors()
    for k, v in res_batched.items():
        res_events[k] = torch.empty_like(v)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    barrier(world)
    torch.cuda.synchronize()
    ev[0].record(stream)
    for _ in range(steps):
        batched()
    ev[1].record(stream)
    torch.cuda.synchronize()
    ev[2].record(stream)
    per_event()
    ev[3].record(stream)
    torch.cuda.synchronize()
    scene.sync_errors()
    identical = all(bool(torch.equal(res_batched[k], res_events[k])) for k in outs)
    ms_b = max_over_ranks(ev[0].elapsed_time(ev[1]) / steps, world)
    ms_e = max_over_ranks(ev[2].elapsed_time(ev[3]), world)
    # (c) one persistent launch whose warps pull photon tiles from a device
    # work queue (tracer fp64_queue), same streams
    res_queue = {}

    def queued():
        return scene.propagate(dev, cfg, engine.Philox(11), outputs=outs, sync=False,
                               results=res_queue, tracer="fp64_queue")
    queued()
    torch.cuda.synchronize()
    ev[0].record(stream)
    for _ in range(steps):
        queued()
    ev[1].record(stream)
    torch.cuda.synchronize()
    scene.sync_errors()
    ms_q = max_over_ranks(ev[0].elapsed_time(ev[1]) / steps, world)
    identical_q = all(bool(torch.equal(res_batched[k], res_queue[k])) for k in outs)
    hit = float((res_batched["sensor"] >= 0).float().mean())
    scene.close()
    del dev, res_batched, res_events, res_queue
    torch.cuda.empty_cache()
    return {"value": n * world / (ms_b * 1e-3), "unit": "photons/s", "ms_per_step": ms_b,
            "photons_per_step_per_gpu": n, "events": int(len(sizes)), "steps": steps,
            "tuning": tuning, "fraction_on_lixels": hit,
            "one_call_per_event": {"value": n * world / (ms_e * 1e-3), "unit": "photons/s",
                                   "ms": ms_e, "calls": int(len(sizes))},
            "persistent_work_queue": {"value": n * world / (ms_q * 1e-3), "unit": "photons/s",
                                      "ms": ms_q, "identical_results": identical_q},
            "batched_over_per_event": ms_e / ms_b, "identical_results": identical}


def run_bunches(args, world, rank, local):
    import torch
    from merlict_development_kit_b200 import factories as F

    torch.cuda.set_device(local)
    flat = F.light_field_telescope(**SCENE).flatten()
    clocks = ClockSampler(local)
    clocks.start()
    form = bunches_form(flat, args.events, args.steps, args.warmup, world, rank, local)
    clk = clocks.stop()
    if rank == 0:
        print(json.dumps({
            "metric": "photons/s", "value": form["value"], "unit": "photons/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": form["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{args.events} air-shower-like events, log-uniform 1e2-1e6 "
                                   "photons, on the light-field telescope (config 2)",
                       "photons_per_step_per_gpu": form["photons_per_step_per_gpu"],
                       "events": form["events"], "max_interactions": MAX_INTERACTIONS,
                       "tuning": form["tuning"],
                       "fraction_on_lixels": form["fraction_on_lixels"]},
            "one_call_per_event": form["one_call_per_event"],
            "persistent_work_queue": form["persistent_work_queue"],
            "batched_over_per_event": form["batched_over_per_event"],
            "identical_results": form["identical_results"],
            "clocks": clk,
        }), flush=True)


def run_signal(args, world, rank, local):
    """The signal chain after binning, one event per step: the photons of a
    config-1 batch that reached lixels (propagated once, untimed) go through
    the night-sky background, photo-electric conversion and pulse
    extraction of all 63,379 lixels (mlgpu_signal_chain), each step with
    its own Philox key.  The CPU baseline is merlict's own chain (one core,
    its Mt19937) on the same photons."""
    import torch
    from merlict_development_kit_b200 import engine, factories as F, signal_chain as SC
    from merlict_development_kit_b200.scenery import Func1

    torch.cuda.set_device(local)
    dev = torch.device(f"cuda:{local}")
    scene_py = F.light_field_telescope(**SCENE)
    scene = engine.Scene(scene_py.flatten())
    n_in = args.event_photons
    ph = engine.photons_to_device(make_photons(n_in, 17 + rank))
    out = scene.propagate(ph, engine.PropagationConfig(MAX_INTERACTIONS), engine.Philox(5 + rank),
                          outputs=("sensor", "time"))
    sensor = out["sensor"].contiguous()
    time_ = out["time"].to(torch.float64).contiguous()
    wavelength = ph["wavelength"].to(torch.float64).contiguous()
    truth = ph["id"].to(torch.int32).contiguous()
    g = F.LightFieldSensorGeometry(F.LightFieldSensorConfig(
        expected_imaging_system_focal_length=SCENE["focal_length"],
        expected_imaging_system_max_aperture_radius=SCENE["aperture_radius"],
        max_FoV_diameter=np.deg2rad(SCENE["fov_deg"]),
        pixel_FoV_hex_flat2flat=np.deg2rad(SCENE["pixel_fov_deg"]),
        num_paxel_on_pixel_diagonal=SCENE["paxels_on_diagonal"],
        housing_overhead=SCENE["housing_overhead"],
        lens_refraction=Func1([[200e-9, 1.5], [1200e-9, 1.5]]),
        bin_reflection=Func1([[200e-9, 0.9], [1200e-9, 0.9]])))
    nl = g.num_lixels
    eff = torch.as_tensor(np.random.default_rng(3).uniform(0.3, 0.7, nl).astype(np.float32),
                          device=dev)
    light = SC.NightSkyBackgroundLight(g, Func1(SIGNAL["nsb_flux"]))
    cfg = SC.SignalChainConfig(
        SC.PhotoElectricConverterConfig(Func1(SIGNAL["qe"]), SIGNAL["dark_rate"],
                                        SIGNAL["crosstalk"]),
        light, SIGNAL["exposure"], SIGNAL["time_slice"], SIGNAL["time_std"])
    n = int(sensor.numel())
    on_lixels = int((sensor >= 0).sum())
    stream = torch.cuda.current_stream()
    for w in range(args.warmup):
        SC.run(scene, cfg, sensor, time_, wavelength, truth, eff, engine.Philox(1000 + w))
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    clocks = ClockSampler(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    ev[0].record(stream)
    pulses = 0
    for k in range(args.steps):
        ps = SC.run(scene, cfg, sensor, time_, wavelength, truth, eff, engine.Philox(k))
        pulses += len(ps.arrival_time_slice)
    ev[1].record(stream)
    torch.cuda.synchronize()
    # end to end: host photon arrays in, the photon stream out, every event
    host = [t.cpu().pin_memory() for t in (sensor, time_, wavelength, truth)]
    dev_bufs = [torch.empty_like(t, device=dev) for t in host]
    barrier(world)
    torch.cuda.synchronize()
    ev[2].record(stream)
    d2h = 0
    for k in range(args.steps):
        for d, h in zip(dev_bufs, host):
            d.copy_(h, non_blocking=True)
        ps = SC.run(scene, cfg, *dev_bufs, eff, engine.Philox(k))
        res = [ps.channel_offset.cpu(), ps.arrival_time_slice.cpu(), ps.simulation_truth_id.cpu()]
        d2h = sum(r.numel() * r.element_size() for r in res)
    ev[3].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(ev[0].elapsed_time(ev[1]) / args.steps, world)
    ms_e2e = max_over_ranks(ev[2].elapsed_time(ev[3]) / args.steps, world)
    h2d = sum(h.numel() * h.element_size() for h in host)
    line = {
        "metric": "photons/s", "value": n * world / (ms * 1e-3), "unit": "photons/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "signal chain after binning of one config-1 event: night-sky "
                               "background, photo-electric conversion and pulse extraction of "
                               f"{nl} lixels", "photons_per_event": n,
                   "photons_on_lixels": on_lixels, "pulses_per_event": pulses / args.steps,
                   "signal": SIGNAL, "inputs_larger_than_l2": n * 24 > 126e6},
        "events_per_s": world / (ms * 1e-3),
        "e2e": {"value": n * world / (ms_e2e * 1e-3), "unit": "photons/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": 8 * args.steps,
        "clocks": clk,
    }
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle as O
        if O.harness_available():
            # the whole event: the chain's per-lixel work (background, dark
            # pulses of all lixels) does not shrink with a photon sample
            take = torch.nonzero(sensor >= 0).flatten()
            r = O.signal_chain_reference(
                1, 1, 0, sensor[take].cpu().numpy(), time_[take].cpu().numpy(),
                wavelength[take].cpu().numpy(), truth[take].cpu().numpy(), nl, eff.cpu().numpy(),
                SIGNAL["qe"], SIGNAL["dark_rate"], SIGNAL["crosstalk"], SIGNAL["nsb_flux"],
                [SCENE["focal_length"], SCENE["aperture_radius"], SCENE["fov_deg"],
                 SCENE["pixel_fov_deg"], SCENE["paxels_on_diagonal"], SCENE["housing_overhead"]],
                SIGNAL["exposure"], SIGNAL["time_slice"], SIGNAL["time_std"])
            line["cpu_baseline"] = {
                "value": n / r["seconds"], "unit": "photons/s", "cores": 1, "kind": "reference",
                "sample": f"merlict's chain (get_photon_pipelines, inject_nsb_into_photon_pipeline,"
                          f" Converter, extract_pulses; Mt19937) on the same event ({len(take)} "
                          f"lixel photons of {n}, all {nl} lixels): {r['seconds']:.3f} s"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    scene.close()


def precision_form(n: int, steps: int, warmup: int, world: int, rank: int, local: int):
    """Precision study (config 3): the large parabolic reflector (0.9 m facets
    of curvature radius 213 m on a 35.5 m aperture) with 8,443 flat pixels at
    106.5 m; photons within 3.5 degrees of the axis.  Photons/s of each form
    and its errors against the FP64 tracer, photon by photon."""
    import torch
    from merlict_development_kit_b200 import engine, factories as F, photons as P, precision

    flat = F.large_reflector_camera().flatten()
    ph = P.downward_disc_source_device(n, 303 + rank, 40.0, 110.0, 3.5, device=f"cuda:{local}",
                                       dtype=torch.float32)
    scene = engine.Scene(flat)
    cfg = engine.PropagationConfig(5)
    rates = {}
    for form in ("fp64", "fp32", "fp32_pure"):
        dt = torch.float32 if form.startswith("fp32") else torch.float64
        planes = {k: v.to(dt) for k, v in ph.items()}
        res = {}
        for _ in range(warmup):
            scene.propagate(planes, cfg, engine.Philox(5), tracer=form, sync=False, results=res,
                            outputs=("sensor", "x", "y", "time"), out_dtype=dt)
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            scene.propagate(planes, cfg, engine.Philox(5), tracer=form, sync=False, results=res,
                            outputs=("sensor", "x", "y", "time"), out_dtype=dt)
        e1.record()
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1) / steps, world)
        rates[form] = n * world / (ms * 1e-3)
        del planes, res
    scene.close()
    errors = precision.study(flat, ph, seed=9, max_interactions=5)
    del ph
    torch.cuda.empty_cache()
    return {"value": rates["fp32"], "unit": "photons/s", "photons_per_s": rates,
            "photons_per_step_per_gpu": n, "steps": steps,
            "fp32_over_fp64": rates["fp32"] / rates["fp64"],
            "errors_vs_fp64": errors}


def run_precision(args, world, rank, local):
    import torch
    torch.cuda.set_device(local)
    form = precision_form(args.photons, args.steps, args.warmup, world, rank, local)
    if rank == 0:
        print(json.dumps({
            "metric": "photons/s", "value": form["value"], "unit": "photons/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "precision study: 5,388-facet parabolic reflector, R = 213 m, "
                                   "8,443 pixels at 106.5 m (config 3)",
                       "photons": args.photons, "max_interactions": 5},
            "photons_per_s": form["photons_per_s"], "errors_vs_fp64": form["errors_vs_fp64"],
        }), flush=True)


def run_calibration(args, world, rank, local):
    """merlict's plenoscope calibration (Calibrator::run_calibration,
    Calibrator.cpp:145-168) of the config-1 light-field telescope: one step =
    `--calibration-photons` calibration photons (8e6, calibration/Config.cpp:
    8-9) generated, propagated (5 interactions) and reduced to every lixel's
    statistics, through calibration.calibrate (the statistics come back to the
    host).  Beside it: the statistics kernel alone (mlgpu_lixel_statistics) on
    per-photon results of the same size, and merlict's own
    LixelStatisticsFiller on the same arrays on one host core."""
    import numpy as np
    import torch
    from merlict_development_kit_b200 import calibration as CAL, engine, factories as F

    torch.cuda.set_device(local)
    flat = F.light_field_telescope(**SCENE).flatten()
    scene = engine.Scene(flat)
    n = args.calibration_photons
    fov_radius = np.deg2rad(SCENE["fov_deg"]) / 2.0
    clocks = ClockSampler(local)

    def step(seed):
        return CAL.calibrate(scene, SCENE["aperture_radius"], fov_radius, num_photons=n,
                             seed=seed)
    for w in range(args.warmup):
        step(100 + w)
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for s in range(args.steps):
        st = step(1 + s)
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    eff = st["efficiency"]
    # the statistics kernel alone, on per-photon results of the same size
    rng = np.random.default_rng(5)
    sensor = rng.integers(-1, flat.num_sensors, size=n).astype(np.int32)
    sensor[rng.random(n) < 0.4] = -1
    vals = [rng.normal(size=n).astype(np.float32) * s_ for s_ in (0.02, 0.02, 2.0, 2.0, 3e-9)]
    dev = [torch.as_tensor(v, device="cuda") for v in [sensor] + vals]
    per_lixel = n / flat.num_sensors
    CAL.lixel_statistics(scene, *dev, per_lixel)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        got = CAL.lixel_statistics(scene, *dev, per_lixel)
    e1.record()
    torch.cuda.synchronize()
    stats_ms = e0.elapsed_time(e1) / args.steps
    ref = None
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        if O.harness_available():
            t0 = time.perf_counter()
            r = O.lixel_statistics_reference(sensor, *vals, flat.num_sensors, 1, n)
            ref_s = time.perf_counter() - t0
            g = np.stack([got[f] for f in CAL.FIELDS], axis=1)
            ref = {"value": n / ref_s, "unit": "photons/s", "cores": 1, "kind": "reference",
                   "sample": f"merlict's LixelStatisticsFiller on the same {n} per-photon results",
                   "identical_to_device": bool(np.array_equal(g, r, equal_nan=True))}
    scene.close()
    if rank == 0:
        print(json.dumps({
            "metric": "photons/s", "value": n / (ms * 1e-3), "unit": "photons/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "plenoscope calibration of the light-field telescope "
                                   "(63,379 lixels): photons, propagation, lixel statistics",
                       "photons_per_step": n, "max_interactions": 5,
                       "lixels_seen": int(np.sum(eff > 0))},
            "lixel_statistics_kernel": {"ms": stats_ms, "photons_per_s": n / (stats_ms * 1e-3)},
            "cpu_baseline": ref, "clocks": clk,
        }), flush=True)


def run_corsika(args, world, rank, local):
    """merlict's EventIoPhotonFactory (merlict_corsika/PhotonFactory.cpp:
    8-136) on the device: one step = `--bunches` CORSIKA photon bunches
    (resident in HBM; weights uniform in [0, 16], a seventh of them whole)
    expanded into photons by mlgpu_corsika_photons, which returns the
    photon count to the host.  The bound is HBM: 32 bytes in per bunch, 60
    bytes out per photon (seven FP64 planes and the bunch id).  Beside it:
    merlict's own factory on a sample of the bunches on one host core."""
    import numpy as np
    import torch
    from merlict_development_kit_b200 import engine, factories as F

    torch.cuda.set_device(local)
    flat = F.light_field_telescope(**SCENE).flatten()
    scene = engine.Scene(flat)
    n = args.bunches
    rng = np.random.default_rng(3)
    b = np.zeros((n, 8), np.float32)
    b[:, 0] = rng.uniform(-15000, 15000, n)
    b[:, 1] = rng.uniform(-15000, 15000, n)
    th = np.deg2rad(rng.uniform(0, 4, n))
    ph = rng.uniform(0, 2 * np.pi, n)
    b[:, 2] = np.sin(th) * np.cos(ph)
    b[:, 3] = np.sin(th) * np.sin(ph)
    b[:, 4] = rng.normal(0, 5, n)
    b[:, 5] = rng.uniform(5e5, 2e6, n)
    w = rng.uniform(0, 16, n)
    w[::7] = np.floor(w[::7])
    b[:, 6] = w
    b[:, 7] = rng.uniform(-700, -250, n)
    bunches = torch.as_tensor(b, device="cuda")
    clocks = ClockSampler(local)
    for wu in range(args.warmup):
        out = scene.corsika_photons(bunches, engine.Philox(wu))
    del out
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    total = 0
    for s in range(args.steps):
        out = scene.corsika_photons(bunches, engine.Philox(10 + s))
        total += int(out["id"].numel())
        del out
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    photons = total / args.steps
    moved = 32.0 * n + 60.0 * photons
    peaks = {}
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            peaks = json.load(f)
    peak = peaks.get("hbm_gbs", 6650.0)
    ref = None
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        if O.harness_available():
            m = min(n, 500_000)
            u = rng.random(m)
            t0 = time.perf_counter()
            r = O.corsika_photons_reference(b[:m], u)
            ref_s = time.perf_counter() - t0
            ref = {"value": r["id"].size / ref_s, "unit": "photons/s", "cores": 1,
                   "kind": "reference",
                   "sample": f"merlict's EventIoPhotonFactory on the first {m} bunches"}
    scene.close()
    if rank == 0:
        print(json.dumps({
            "metric": "photons/s", "value": photons / (ms * 1e-3), "unit": "photons/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "CORSIKA photon bunches expanded on the device",
                       "bunches_per_step": n, "photons_per_step": photons},
            "roofline": {"bound": "hbm", "achieved": moved / (ms * 1e-3) / 1e9,
                         "peak": peak, "unit": "GB/s",
                         "frac": moved / (ms * 1e-3) / 1e9 / peak,
                         "algorithmic_bytes": "32 per bunch + 60 per photon",
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs"},
            "cpu_baseline": ref, "clocks": clk,
        }), flush=True)


def run_surrogate(args, world, rank, local):
    """The learned surrogate (config 4) on the light-field telescope: trained
    on `--train-photons` photons traced exactly (FP64), evaluated on
    `--photons` fresh photons against exact tracing of the same photons:
    photons/s of both, per-lixel Jensen-Shannon divergence, fraction of
    photons traced exactly by fallback, and the tensor-core throughput."""
    import torch
    from merlict_development_kit_b200 import engine, factories as F, surrogate as S

    torch.cuda.set_device(local)
    flat = F.light_field_telescope(**SCENE).flatten()
    scene = engine.Scene(flat)
    src = S.Source(SOURCE["disc_radius"], SOURCE["height"], SOURCE["max_zenith_deg"])
    plane = args.surrogate_mode == "plane"
    plane_z = SCENE["focal_length"] - 0.05   # 5 cm below the lens array
    t0 = time.perf_counter()
    if plane:
        data = S.training_data_plane(scene, src, args.train_photons, seed=1 + rank,
                                     plane_z=plane_z)
    else:
        data = S.training_data(scene, src, args.train_photons, seed=1 + rank,
                               max_interactions=MAX_INTERACTIONS)
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    model = S.Surrogate(flat, source=src, seed=rank, plane_z=plane_z if plane else None)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    losses = model.train(data, epochs=args.epochs, batch=65536, lr=2e-3)
    e1.record()
    torch.cuda.synchronize()
    train_s = e0.elapsed_time(e1) * 1e-3
    trained = (args.train_photons // 65536) * 65536 * args.epochs
    del data
    n = args.photons
    ph = src.photons(n, seed=777 + rank)
    cfg = engine.PropagationConfig(MAX_INTERACTIONS)

    tuning, _ = scene.autotune({k: v[:2_000_000].contiguous() for k, v in ph.items()}, cfg,
                               engine.Philox(3))

    def exact():
        return scene.propagate(ph, cfg, engine.Philox(4242), outputs=("sensor",),
                               tuning=tuning)["sensor"]

    def learned(use_network=True):
        return model.propagate(ph, seed=99, scene=scene, max_interactions=MAX_INTERACTIONS,
                               use_network=use_network)

    def hist(sn):
        sn = sn[sn >= 0].long()
        return torch.bincount(sn, minlength=flat.num_sensors).double().cpu().numpy()
    from merlict_development_kit_b200.precision import js_divergence
    r_exact = exact()
    h_exact = hist(r_exact)
    # operating point: the widest component (in units of the smallest lixel's
    # inner radius) that still keeps the per-lixel JS within the target
    # the unit of the fallback threshold: the smallest lixel's inner radius
    # (lookup mode) or 1 mm on the plane (plane mode)
    unit = model.grid.inner_min if model.grid is not None else 1e-3
    sweep = []
    for mult in (0.0625, 0.25, 1.0, 4.0, 16.0, 64.0):
        r = model.propagate(ph, seed=99, scene=scene, max_interactions=MAX_INTERACTIONS,
                            sigma_limit=mult * unit, tuning=tuning)
        sweep.append({"sigma_limit_m": mult * unit,
                      "js": js_divergence(hist(r["sensor"]), h_exact),
                      "fallback": float(r["fallback"].float().mean())})
    ok = [s_ for s_ in sweep if s_["js"] <= args.js_target]
    chosen = (max(ok, key=lambda s_: s_["sigma_limit_m"]) if ok
              else min(sweep, key=lambda s_: s_["js"]))
    limit = chosen["sigma_limit_m"]

    def learned(use_network=True):
        return model.propagate(ph, seed=99, scene=scene, max_interactions=MAX_INTERACTIONS,
                               use_network=use_network, sigma_limit=limit, tuning=tuning)

    learned()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record()
    r_net = learned()
    ev[1].record()
    r_exact = exact()
    ev[2].record()
    torch.cuda.synchronize()
    ms_net, ms_exact = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])
    # the network alone: forward pass of one chunk on the tensor cores
    x = src.inputs({k: v[:1 << 22] for k, v in ph.items()})
    model.forward(x)
    ev[2].record()
    for _ in range(5):
        model.forward(x)
    ev[3].record()
    torch.cuda.synchronize()
    fwd_ms = ev[2].elapsed_time(ev[3]) / 5
    tc_flops = 2.0 * (128 * 256 + 3 * 256 * 256 + 256 * 80) * x.shape[0]   # tensor-core layers
    r_null = model.propagate(ph, seed=99, use_network=False, sigma_limit=1e9)
    js_net = js_divergence(hist(r_net["sensor"]), h_exact)
    js_null = js_divergence(hist(r_null["sensor"]), h_exact)
    # the noise floor: two exact runs with independent streams
    r_exact2 = scene.propagate(ph, cfg, engine.Philox(4243), outputs=("sensor",))["sensor"]
    js_floor = js_divergence(hist(r_exact2), h_exact)
    peaks = {}
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            peaks = json.load(f)
    peak_tf = peaks.get("bf16_tflops", 1590.0)
    achieved = tc_flops / (fwd_ms * 1e-3) / 1e12
    if rank == 0:
        print(json.dumps({
            "metric": "photons/s", "value": n / (ms_net * 1e-3), "unit": "photons/s",
            "n_gpus": world, "steps": 1, "warmup": 1, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16", "data": "synthetic",
            "config": {"workload": "learned surrogate on the light-field telescope (config 4)",
                       "mode": args.surrogate_mode,
                       "train_photons": args.train_photons, "epochs": args.epochs,
                       "eval_photons": n, "max_interactions": MAX_INTERACTIONS,
                       "network": "5 inputs (sin/cos-encoded to 128) -256x4 SiLU-73, 8-component "
                                  "mixture, BF16 on tcgen05"},
            "exact_fp64": {"value": n / (ms_exact * 1e-3), "unit": "photons/s"},
            "speedup_over_exact": ms_exact / ms_net,
            "lixel_js": {"surrogate": js_net, "without_network": js_null,
                         "two_exact_runs": js_floor},
            "fallback_fraction": float(r_net["fallback"].float().mean()),
            "sigma_limit_m": limit, "js_target": args.js_target, "sweep": sweep,
            "training": {"loss_per_epoch": losses, "seconds": train_s,
                         "photons_per_s": trained / train_s, "trace_seconds": t_data},
            "roofline": {"bound": "tensor", "kernel": "tensor-core layers (forward)",
                         "achieved": achieved, "peak": peak_tf, "unit": "TFLOP/s",
                         "frac": achieved / peak_tf, "forward_ms_per_4Mi": fwd_ms,
                         "peak_source": "measured MEASURED_PEAKS.json bf16_tflops"
                         if "bf16_tflops" in peaks else "fallback"},
        }), flush=True)
    scene.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--tracer", choices=["fp64", "fp64_plain", "fp32"], default="fp64")
    ap.add_argument("--photons", type=int, default=10_000_000)
    ap.add_argument("--ref-photons", type=int, default=100_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the FP32 form's line items in the default workload")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="default wavefront knobs instead of mlgpu_scene_autotune's")
    ap.add_argument("--workload", choices=["telescope", "bunches", "precision", "surrogate",
                                           "signal", "calibration", "corsika"],
                    default="telescope",
                    help="telescope: the light-field telescope batch; bunches: 4096 "
                         "air-shower-like events of uneven sizes, batched vs one call per event; "
                         "precision: the FP32 forms against FP64 on the large reflector; "
                         "signal: the signal chain after binning of one config-1 event; "
                         "calibration: the plenoscope calibration (8e6 photons); "
                         "corsika: CORSIKA bunches expanded into photons on the device")
    ap.add_argument("--calibration-photons", type=int, default=8_000_000)
    ap.add_argument("--bunches", type=int, default=8_000_000)
    ap.add_argument("--events", type=int, default=4096)
    ap.add_argument("--precision-photons", type=int, default=100_000_000,
                    help="photons of the precision study (config 3) in the default line's forms")
    ap.add_argument("--event-photons", type=int, default=1_000_000,
                    help="photons of the event the signal workload propagates once")
    ap.add_argument("--train-photons", type=int, default=200_000_000)
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--js-target", type=float, default=1e-3)
    ap.add_argument("--surrogate-mode", choices=["plane", "lookup"], default="plane",
                    help="plane: the network models the photon 5 cm below the lens array and the "
                         "exact tracer carries it through the light-field sensor; lookup: the "
                         "network models the final hit and the lixel is looked up")
    args = ap.parse_args()
    world, rank, local = init_dist()
    try:
        if args.impl == "reference":
            run_reference_arm(args, world, rank)
        elif args.workload == "bunches":
            run_bunches(args, world, rank, local)
        elif args.workload == "precision":
            run_precision(args, world, rank, local)
        elif args.workload == "surrogate":
            run_surrogate(args, world, rank, local)
        elif args.workload == "signal":
            run_signal(args, world, rank, local)
        elif args.workload == "calibration":
            run_calibration(args, world, rank, local)
        elif args.workload == "corsika":
            run_corsika(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            if dist.is_initialized():
                dist.destroy_process_group()


if __name__ == "__main__":
    main()
