#!/usr/bin/env python
"""bench.py — throughput of the sm_100a wavefront path tracer (libpt).

Workload (default): 64 UV spheres of 20,480 triangles (1,310,720 triangles)
on an 8 x 8 grid with Disney parameters drawn U[0,1] (roughness U[0.05,1]),
a procedural 2048 x 1024 float32 sky + sun envmap (peak 5e4), 1280 x 720,
64 samples per pixel, depth 16, MIS.  One step = one 64-spp frame
(58,982,400 paths).  Synthetic, seeded inputs stand in for the reference's
scene assets.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl pt|reference]

Each rank renders its own 64-spp frame from a disjoint sample-index range and
the films are summed with one NCCL all-reduce per step (weak scaling).  The
value is the whole-job paths per second (device time, CUDA events on libpt's
stream, max over ranks).  `e2e` repeats the measurement through pt_render with
pinned host films (copies inside the timed region).  `--impl reference` times
the reference's own shader code compiled for the CPU (oracle/_ref/libref.so,
else the oracle restatement) on the host cores.
"""

from __future__ import annotations

import argparse
import ctypes as C
import importlib
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "pbrt-renderer-_b200")
sys.path.insert(0, ROOT)

METRIC = "Mpaths/s and time-to-relMSE 1e-2, cached vs plain PT on one B200"
BYTES_PER_EXT_RAY = 48    # ray in (o, d, tmin, tmax: 32 B) + hit out (t, prim, u, v: 16 B)
BYTES_PER_SHADOW_RAY = 36  # ray in (32 B) + visibility out (4 B)
BYTES_PER_PATH_FILM = 64   # float4 sum + float4 Kahan compensation read-modify-write


def load_pkg():
    if "pbrt_b200" in sys.modules:
        return sys.modules["pbrt_b200"]
    spec = importlib.util.spec_from_file_location("pbrt_b200", os.path.join(PKG, "__init__.py"),
                                                  submodule_search_locations=[PKG])
    m = importlib.util.module_from_spec(spec)
    sys.modules["pbrt_b200"] = m
    spec.loader.exec_module(m)
    return m


def workload(name, scale=1.0):
    pt = load_pkg()
    scenes = importlib.import_module("pbrt_b200.scenes")
    if name == "disney_envmap":
        W, H, spp, depth = 1280, 720, 64, 16
        sc, cam = scenes.disney_spheres(W, H)
        cfg = {"workload": "disney_envmap", "spheres": 64, "triangles": sc.num_triangles, "width": W, "height": H,
               "spp": spp, "max_depth": depth, "envmap": "2048x1024 rgb32f", "mis": True}
    elif name == "cornell":
        W, H, spp, depth = 256, 256, 16, 8
        sc, cam = scenes.cornell(W, H)
        cfg = {"workload": "cornell", "triangles": sc.num_triangles, "width": W, "height": H, "spp": spp,
               "max_depth": depth}
    elif name == "radiance_cache":
        W, H, spp, depth = 1920, 1080, 16, 16
        sc, cam = scenes.radiance_cache_scene(W, H)
        cfg = {"workload": "radiance_cache", "triangles": sc.num_triangles, "instances": 122, "width": W, "height": H,
               "spp": spp, "max_depth": depth, "materials": "Disney + hair (every 7th instance)",
               "medium": "homogeneous fog box, albedo 0.9, g 0.3", "envmap": "2048x1024 rgb32f"}
    elif name == "hair_volume":
        W, H, spp, depth = 1024, 1024, 128, 16
        sc, cam = scenes.hair_volume(W, H)
        cfg = {"workload": "hair_volume", "triangles": sc.num_triangles, "width": W, "height": H, "spp": spp,
               "max_depth": depth, "grid": "128^3 fbm"}
    else:
        raise SystemExit(f"unknown workload {name}")
    return pt, sc, cam, W, H, spp, depth, cfg


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in self.rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# k_extend DRAM traffic per extension ray (dram__bytes_read.sum + dram__bytes_write.sum
# from one ncu capture of this workload at 8 spp, the smallest case in the
# grouped path order (groups of 8 samples): 383.3 MB over the 7,372,800
# camera rays of bounce 0; the full frame's groups of 32 are more coherent,
# so this is an upper bound for it).  The scene is L2-resident and the
# queues stream once, so traffic scales with the rays a launch processes.
EXTEND_DRAM_BYTES_PER_RAY = {"disney_envmap": 52.0}


REF_SPP = 4096        # reference image: plain path tracing, samples [0, 4096)
TTQ_TARGET = 1e-2     # relMSE bar
TTQ_OFFSET = 1 << 20  # progressive renders draw samples from here on (independent of the reference)
# relMSE is checked at accumulated spp ~ 2^(k/2) (both forms, same points)
TTQ_CHECKS = sorted({int(round(2 ** (k / 2))) for k in range(0, 21)})


def relmse(x, ref):
    """mean((x - ref)^2 / (ref^2 + 1e-2)) over pixels and RGB, the relMSE of
    the reference's comparison tool (validation_tests/compare_exr.py:102)."""
    return float(((x - ref) ** 2 / (ref ** 2 + 1e-2)).mean())


def reference_image(pt, ctx, W, H, cam, depth, env_mode, chunk):
    """The 4096-spp plain render (samples [0, 4096)) both forms are scored against."""
    D = importlib.import_module("pbrt_b200.distributed")
    ref = D.new_film(H, W, device="cuda")
    for k in range(REF_SPP // chunk):
        P = pt.render_params(W, H, chunk, cam, max_depth=depth, sample_offset=k * chunk, env_sampling=env_mode)
        ctx.render(P, ref[0].data_ptr(), ref[1].data_ptr(), pt.PT_MEM_DEVICE)
    return D.resolve(ref)


def progressive(pt, ctx, stream, W, H, ref_img, make_params, spf, warm=0):
    """Progressive accumulation (the reference's frame-by-frame accumulation):
    render calls of `spf` samples, the first `warm` of them into a discarded
    film (cache training only), each call's device time from libpt's CUDA
    events around its launches (pt_stats.ms_total: the render, its cache
    inference and training; not the one-time capture of a launch graph for a
    new call shape).  relMSE against ref_img at the TTQ_CHECKS points (outside the
    timing); the first point at or below the bar gives the time."""
    import torch

    D = importlib.import_module("pbrt_b200.distributed")
    film = D.new_film(H, W, device="cuda")
    scratch = D.new_film(H, W, device="cuda") if warm else None
    calls, acc, total_ms, curve, reached = 0, 0, 0.0, [], None
    checks = [c for c in TTQ_CHECKS if c >= spf]
    while acc < REF_SPP // 4:
        P = make_params(TTQ_OFFSET + calls * spf)
        tgt = scratch if calls < warm else film
        _, _, st = ctx.render(P, tgt[0].data_ptr(), tgt[1].data_ptr(), pt.PT_MEM_DEVICE)
        total_ms += st.ms_total
        calls += 1
        if calls <= warm:
            continue
        acc += spf
        if checks and acc >= checks[0]:
            while checks and acc >= checks[0]:
                checks.pop(0)
            e = relmse(D.resolve(film), ref_img)
            curve.append([acc, round(e, 6), round(total_ms / 1e3, 5)])
            if e <= TTQ_TARGET:
                reached = (acc, total_ms / 1e3)
                break
    return {"seconds": None if reached is None else round(reached[1], 5),
            "spp": None if reached is None else reached[0], "curve": curve}


# Radiance-cache settings of the cached form: calls of CACHE_CALLS[workload]
# = (spp per call, training-only warm-up calls) from sweeps of each scene (the
# 64-sphere scene: 8-spp calls after 3; the 10 M-triangle fogged scene: 4-spp
# calls after 8), 4 training steps per call, up to 65,536 records per call
# from at most 10 % of the paths that reach a cache vertex, bounces with
# Disney roughness >= 0.1 end into the cache, no unbiased suffixes; inference
# uses an exponential average of the weights (decay 0.97), which removes the
# frame-to-frame flicker of a cache that takes 4 steps per call.
CACHE_RECORDS, CACHE_LR, CACHE_EMA = 65536, 1e-2, 0.97
CACHE_CALLS = {"disney_envmap": (8, 3), "radiance_cache": (4, 8)}
CACHE_CALLS_DEFAULT = (4, 8)
CACHE_FRACTION, CACHE_ROUGH = 0.1, 0.1


TTQ_RANGE_STRIDE = 1 << 22  # repeated runs draw from sample ranges this far apart (each uses < 2^11 spp)


def _summary(runs):
    """Median and worst (slowest) of repeated time-to-relMSE runs; None
    entries (the bar not reached) count as slowest."""
    secs = [r["seconds"] for r in runs]
    reached = sorted(x for x in secs if x is not None)
    out = {"runs": len(runs), "reached": len(reached), "seconds_each": secs, "spp_each": [r["spp"] for r in runs]}
    if len(reached) == len(runs):
        out["seconds"] = round(float(np.median(reached)), 5)
        out["worst_seconds"] = round(reached[-1], 5)
    else:
        out["seconds"] = round(float(np.median(reached)), 5) if len(reached) * 2 > len(runs) else None
        out["worst_seconds"] = None
    out["spp"] = runs[0]["spp"]
    out["curve"] = runs[0]["curve"]  # the first run's relMSE curve
    return out


def time_to_relmse(pt, ctx, stream, W, H, cam, depth, env_mode, chunk, calls=CACHE_CALLS_DEFAULT, seeds=(0, 1, 2),
                   plain_runs=3):
    """Device time for plain and radiance-cached path tracing to reach relMSE
    <= 1e-2 against a 4096-spp plain render of the same scene, checked at
    accumulated spp 1, 2, 3, 4, 6, 8, 11, ... (~2^(k/2)) in both forms.
    Plain: one render call per check point (calls grow with it).  Cached:
    calls[0]-spp calls with training steps in each, the first calls[1] of
    them training only, from an untrained cache (training time and the
    warm-up calls are inside the timed total).  Repeated: plain over
    `plain_runs` independent sample ranges, cached over the training seeds
    `seeds`, each with its own sample range; median and worst reported."""
    spf, warm_calls = calls
    ref_img = reference_image(pt, ctx, W, H, cam, depth, env_mode, chunk)
    D = importlib.import_module("pbrt_b200.distributed")
    import torch

    def plain_run(offset):
        film = D.new_film(H, W, device="cuda")
        done, total_ms, curve, reached = 0, 0.0, [], None
        for nxt in TTQ_CHECKS:
            add = nxt - done
            P = pt.render_params(W, H, add, cam, max_depth=depth, sample_offset=offset + done, env_sampling=env_mode)
            _, _, st = ctx.render(P, film[0].data_ptr(), film[1].data_ptr(), pt.PT_MEM_DEVICE)
            total_ms += st.ms_total
            done += add
            e = relmse(D.resolve(film), ref_img)
            curve.append([done, round(e, 6), round(total_ms / 1e3, 5)])
            if e <= TTQ_TARGET:
                reached = (done, total_ms / 1e3)
                break
        return {"seconds": None if reached is None else round(reached[1], 5),
                "spp": None if reached is None else reached[0], "curve": curve}

    def cache_params(seed):
        return pt.cache_params(seed=seed, train_records=CACHE_RECORDS, learning_rate=CACHE_LR, ema=CACHE_EMA,
                               max_train_fraction=CACHE_FRACTION, rough_threshold=CACHE_ROUGH)

    def cached_params(off):
        return pt.render_params(W, H, spf, cam, max_depth=depth, sample_offset=off, env_sampling=env_mode,
                                flags=pt.PT_RENDER_RADIANCE_CACHE)

    plain_list = [plain_run(TTQ_OFFSET + r * TTQ_RANGE_STRIDE) for r in range(plain_runs)]
    # one untimed cached call first: the cache kernels' first launch in the
    # process (module loading, graph instantiation) is set-up, not rendering
    ctx.cache_init(cache_params(0))
    warm = D.new_film(H, W, device="cuda")
    ctx.render(cached_params(0), warm[0].data_ptr(), warm[1].data_ptr(), pt.PT_MEM_DEVICE)
    ctx.cache_release()
    torch.cuda.synchronize()
    cached_list, steps = [], 0
    for i, seed in enumerate(seeds):
        ctx.cache_init(cache_params(seed))
        try:
            base = TTQ_OFFSET + i * TTQ_RANGE_STRIDE
            cached_list.append(progressive(pt, ctx, stream, W, H, ref_img, lambda off: cached_params(base + off), spf,
                                           warm=warm_calls))
            steps = int(ctx.cache_stats().steps)
        finally:
            ctx.cache_release()
    plain, cached = _summary(plain_list), _summary(cached_list)
    cached["seeds"] = list(seeds)
    cached["settings"] = {"spp_per_call": spf, "warmup_calls": warm_calls, "train_records_per_call": CACHE_RECORDS,
                          "max_train_fraction": CACHE_FRACTION, "rough_threshold": CACHE_ROUGH,
                          "learning_rate": CACHE_LR, "ema": CACHE_EMA, "adam_steps_per_run": steps,
                          "network": "64 in, 5 x 64 ReLU, 3 out; BF16 tcgen05, FP32 accumulation"}
    out = {"target": TTQ_TARGET, "reference_spp": REF_SPP, "plain": plain, "cached": cached}
    if plain["seconds"] and cached["seconds"]:
        out["cached_speedup"] = round(plain["seconds"] / cached["seconds"], 3)
        if cached["worst_seconds"]:
            out["cached_speedup_vs_worst_cached"] = round(plain["seconds"] / cached["worst_seconds"], 3)
    elif cached["seconds"] and plain["curve"]:
        # plain did not reach the bar within REF_SPP / 4 samples: its time so far bounds the ratio from below
        out["cached_speedup_at_least"] = round(plain["curve"][-1][2] / cached["seconds"], 3)
        if cached["worst_seconds"]:
            out["cached_speedup_at_least_vs_worst_cached"] = round(plain["curve"][-1][2] / cached["worst_seconds"], 3)
    return out


# Radiance-cache network FLOPs (the MMA shapes: 64 inputs, 5 x 64 hidden,
# output padded to 16): forward per query; training per record adds the
# weight gradients of all 6 layers and the input gradients of layers 5..1.
CACHE_FLOPS_INFER = 2 * (5 * 64 * 64 + 16 * 64)
CACHE_FLOPS_TRAIN = CACHE_FLOPS_INFER + 2 * (5 * 64 * 64 + 16 * 64) + 2 * (16 * 64 + 4 * 64 * 64)


def cache_kernel_roofline(pt, ctx):
    """Tensor-core roofline of the two network kernels on large batches in
    device memory: k_rc_infer over 2^21 queries, k_rc_train over 2^18
    records; device time from the library's CUDA events around the kernel,
    median of 10 calls after 3 warm-up calls; peak = measured dense BF16."""
    import torch

    pk = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    peak = float(pk.get("bf16_tflops", 1590.0))
    L, h = ctx.L, ctx.h
    ctx.cache_init(pt.cache_params(seed=0, bbox=((0, 0, 0), (1, 1, 1))))
    g = torch.Generator(device="cuda").manual_seed(0)
    out = {}
    try:
        for kind, n, flops in (("infer", 1 << 21, CACHE_FLOPS_INFER), ("train", 1 << 18, CACHE_FLOPS_TRAIN)):
            f = torch.rand((n, 64), device="cuda", generator=g) * 2 - 1
            f[:, 49] = 1.0
            f[:, 50:] = 0.0
            fp = C.cast(f.data_ptr(), C.POINTER(C.c_float))
            if kind == "infer":
                y = torch.empty((n, 3), device="cuda")
                yp = C.cast(y.data_ptr(), C.POINTER(C.c_float))
                call = lambda: L.pt_cache_infer_batch(h, fp, n, yp, pt.PT_MEM_DEVICE)  # noqa: E731
            else:
                t = torch.rand((n, 3), device="cuda", generator=g) * 2
                tp = C.cast(t.data_ptr(), C.POINTER(C.c_float))
                gr = np.zeros(pt.PT_CACHE_PARAMS, np.float32)
                loss = np.zeros(1, np.float32)
                call = lambda: L.pt_cache_gradient_batch(h, fp, tp, n, pt.fptr(gr), pt.fptr(loss),  # noqa: E731
                                                         pt.PT_MEM_DEVICE)
            ms = []
            for k in range(13):
                ctx._check(call())
                if k >= 3:
                    ms.append(ctx.cache_stats().last_kernel_ms)
            m = float(np.median(ms))
            tf = n * flops / (m / 1e3) / 1e12
            out[kind] = {"rows": n, "flops_per_row": flops, "ms": round(m, 4), "achieved": round(tf, 2),
                         "peak": peak, "unit": "TFLOP/s", "frac": round(tf / peak, 4)}
    finally:
        ctx.cache_release()
    return out


def _timed_calls(pt, ctx, W, H, make_params, steps, warmup):
    """Device time of `steps` render calls (libpt's events around each call's
    launches) after `warmup` untimed ones, each from its own sample range,
    into a device film; L2 flushed before each timed call."""
    import torch

    D = importlib.import_module("pbrt_b200.distributed")
    film = D.new_film(H, W, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    ms = []
    for k in range(warmup + steps):
        flush.zero_()
        _, _, st = ctx.render(make_params(k), film[0].data_ptr(), film[1].data_ptr(), pt.PT_MEM_DEVICE)
        if k >= warmup:
            ms.append(st.ms_total)
    return ms


def config3_sweep(pt, steps=2, warmup=1):
    """Configuration 3: 20,000 hair strands x 32 segments as camera-facing
    ribbons (1.28 M triangles, Chiang BCSDF, eumelanin U[0.1, 8], beta_m =
    beta_n = 0.3, alpha 2 deg) in a 128^3 fBm density grid (albedo 0.9),
    1024 x 1024, 128 spp, depth 16, for HG g in {0, 0.3, 0.8}; heterogeneous
    media in the wavefront form (PT_RENDER_MEDIA_WAVEFRONT).  Mpaths/s from
    the median device time of `steps` frames."""
    scenes = importlib.import_module("pbrt_b200.scenes")
    W = H = 1024
    spp, depth = 128, 16
    sc, cam = scenes.hair_volume(W, H)
    ctx = pt.Context(0)
    out = {"workload": "hair_volume: 20k strands x 32 segments (1.28 M ribbon triangles), 128^3 fBm medium, "
                       "albedo 0.9, 1024x1024, 128 spp, depth 16, wavefront media", "steps": steps, "g": {}}
    try:
        for g in (0.0, 0.3, 0.8):
            sc.volumes[0].phase_g = g
            ctx.upload(sc)

            def params(k):
                return pt.render_params(W, H, spp, cam, max_depth=depth, sample_offset=k * spp,
                                        flags=pt.PT_RENDER_MEDIA_WAVEFRONT)

            ms = float(np.median(_timed_calls(pt, ctx, W, H, params, steps, warmup)))
            out["g"][str(g)] = {"ms_per_frame": round(ms, 2), "mpaths_per_s": round(W * H * spp / (ms / 1e3) / 1e6, 2)}
    finally:
        ctx.close()
    return out


def config5_run(pt, steps=3, warmup=1):
    """Configuration 5: ~10 M triangles (122 displaced icospheres of 81,920
    triangles on a ground plane and back wall, Disney with every 7th instance
    hair, a homogeneous fog box), 2048 x 1024 sky + sun envmap, 1920 x 1080,
    depth 16: plain Mpaths/s at 16 spp per frame and the cached vs plain time
    to relMSE 1e-2 (three training seeds)."""
    scenes = importlib.import_module("pbrt_b200.scenes")
    W, H, spp, depth = 1920, 1080, 16, 16
    sc, cam = scenes.radiance_cache_scene(W, H)
    ctx = pt.Context(0)
    try:
        ctx.upload(sc)

        def params(k):
            return pt.render_params(W, H, spp, cam, max_depth=depth, sample_offset=k * spp)

        ms = float(np.median(_timed_calls(pt, ctx, W, H, params, steps, warmup)))
        out = {"workload": "radiance_cache: %d triangles, 1920x1080, depth 16, fog box, sky+sun envmap"
                           % sc.num_triangles,
               "plain_16spp": {"ms_per_frame": round(ms, 2), "mpaths_per_s": round(W * H * spp / (ms / 1e3) / 1e6, 2)}}
        import torch

        out["time_to_relmse"] = time_to_relmse(pt, ctx, torch.cuda.current_stream(), W, H, cam, depth, pt.PT_ENV_CDF,
                                               64, calls=CACHE_CALLS["radiance_cache"], plain_runs=1)
    finally:
        ctx.close()
    return out


def cache_render_roofline(pt, ctx, W, H, cam, depth, env_mode, spp=8):
    """Tensor-core roofline of the network kernels as the cached form runs
    them: the render-mode inference (queries encoded from path records,
    Lo += throughput x cache) and training (the call's records, 4 steps)
    inside a cached render of the workload, timed by libpt's events around
    those launches (PT_RENDER_STAGE_TIMING); three untimed cached calls first
    so the cache has trained."""
    import torch

    D = importlib.import_module("pbrt_b200.distributed")
    pk = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    peak = float(pk.get("bf16_tflops", 1590.0))
    ctx.cache_init(pt.cache_params(seed=0, train_records=CACHE_RECORDS, learning_rate=CACHE_LR, ema=CACHE_EMA,
                                   max_train_fraction=CACHE_FRACTION, rough_threshold=CACHE_ROUGH))
    film = D.new_film(H, W, device="cuda")
    try:
        for k in range(4):
            P = pt.render_params(W, H, spp, cam, max_depth=depth, sample_offset=k * spp, env_sampling=env_mode,
                                 flags=pt.PT_RENDER_RADIANCE_CACHE | (pt.PT_RENDER_STAGE_TIMING if k == 3 else 0))
            ctx.render(P, film[0].data_ptr(), film[1].data_ptr(), pt.PT_MEM_DEVICE)
        torch.cuda.synchronize()
        st = ctx.cache_stats()
    finally:
        ctx.cache_release()
    out = {"call": f"{W}x{H}, {spp} spp, cached"}
    for kind, rows, ms, flops in (("infer", int(st.queries), st.last_render_infer_ms, CACHE_FLOPS_INFER),
                                  ("train", int(st.last_render_train_rows), st.last_render_train_ms,
                                   CACHE_FLOPS_TRAIN)):
        tf = rows * flops / (ms / 1e3) / 1e12 if ms > 0 else 0.0
        out[kind] = {"rows": rows, "flops_per_row": flops, "ms": round(float(ms), 4), "achieved": round(tf, 2),
                     "peak": peak, "unit": "TFLOP/s", "frac": round(tf / peak, 4)}
    return out


BATCH_STEPS = 3


def batched_requests_run(pt):
    """Configuration 4: 32 requests over the Cornell box and the Disney spheres
    (random cameras, sides log-uniform 64..1024, spp U{4..256}).  Each
    scene's requests form one batch (pt_render_batch: one wavefront, one
    captured graph); the two batches run concurrently, each on its own
    context and stream (one host thread per context).  Launch shapes come
    from pt_batch_autotune (untimed); then 1 warm-up and BATCH_STEPS timed
    batch pairs.  Device time per step = the longer batch (both start
    together); per-request latency = device time from its batch's start to
    the end of the wave that finished it."""
    import torch

    scenes = importlib.import_module("pbrt_b200.scenes")
    reqs = scenes.batch_requests(32, seed=0)
    built = {"cornell": scenes.cornell(256, 256)[0], "disney_envmap": scenes.disney_spheres(1280, 720)[0]}
    groups = {}
    for q in reqs:
        groups.setdefault(q["scene"], []).append(q)
    runs = []
    for name, qs in groups.items():
        ctx = pt.Context(0)
        ctx.upload(built[name])
        params = [pt.render_params(q["width"], q["height"], q["spp"], q["camera"], max_depth=q["max_depth"])
                  for q in qs]
        films = [(torch.zeros((q["height"], q["width"], 4), device="cuda"),
                  torch.zeros((q["height"], q["width"], 4), device="cuda")) for q in qs]
        ptrs = [(a.data_ptr(), b.data_ptr()) for a, b in films]
        tune = ctx.batch_autotune(params, ptrs, pt.PT_MEM_DEVICE)
        runs.append({"name": name, "ctx": ctx, "params": params, "films": films, "ptrs": ptrs, "tune": tune})

    def one(r, off, res):
        for P in r["params"]:
            P.sample_offset = off
        _, ms, st = r["ctx"].render_batch(r["params"], r["ptrs"], pt.PT_MEM_DEVICE)
        res[r["name"]] = (ms, st)

    steps = []
    for k in range(BATCH_STEPS + 1):
        res = {}
        th = [threading.Thread(target=one, args=(r, 1000 * k, res)) for r in runs]
        for t in th:
            t.start()
        for t in th:
            t.join()
        if k:
            steps.append(res)
    paths = sum(P.width * P.height * P.spp for r in runs for P in r["params"])
    step_ms = [max(st.ms_total for _, st in res.values()) for res in steps]
    lat = np.concatenate([ms for res in steps for ms, _ in res.values()])
    out = {
        "workload": "32 requests: cornell 256^2 scene (depth 8) + disney_envmap scene (depth 16), random cameras, "
                    "sides log-uniform 64..1024, spp U{4..256}, seed 0",
        "requests": {r["name"]: len(r["params"]) for r in runs},
        "paths_per_step": int(paths),
        "steps": BATCH_STEPS,
        "ms_per_step": round(float(np.mean(step_ms)), 3),
        "mpaths_per_s": round(paths / (float(np.mean(step_ms)) / 1e3) / 1e6, 2),
        "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 3), "p99": round(float(np.percentile(lat, 99)), 3),
                       "max": round(float(lat.max()), 3)},
        "launches": {r["name"]: int(steps[-1][r["name"]][1].launches) for r in runs},
        "waves": {r["name"]: int(steps[-1][r["name"]][1].waves) for r in runs},
        "autotune": {r["name"]: {"wave_paths": r["tune"].wave_paths, "traversal_grid": r["tune"].traversal_grid,
                                 "candidates": [[int(r["tune"].candidate_wave[i]), float(r["tune"].candidate_grid[i]),
                                                 round(float(r["tune"].candidate_ms[i]), 3)]
                                                for i in range(r["tune"].candidates)]} for r in runs},
    }
    for r in runs:
        r["ctx"].close()
    return out


def cpu_reference_run(pt, sc, cam, W, H, depth, seconds=15.0, prefer_reference=True):
    """Time the CPU implementation on a bounded sample of the workload:
    whole frames at 1 spp (the reference's one-sample dispatch), repeated
    until about `seconds` of work; returns (Mpaths/s, kind, cores, sample)."""
    from oracle.oracle import Oracle, Reference
    cores = os.cpu_count() or 1
    if prefer_reference and Reference.available():
        impl, kind = Reference(pt), "reference"
    else:
        impl, kind = Oracle(pt), "port"
    impl.load(sc)
    frames, t_total, paths = 0, 0.0, 0
    rows = H
    while t_total < seconds and frames < 1024:
        P = pt.render_params(W, rows, 1, cam, max_depth=depth, sample_offset=frames)
        t0 = time.perf_counter()
        if kind == "reference":
            impl.render(P, threads=cores)
        else:
            impl.render(P, threads=cores)
        dt = time.perf_counter() - t0
        t_total += dt
        paths += W * rows
        frames += 1
    accel = ("ray queries on a binned-SAH BVH with the cost model of the reference's CPU accelerator "
             "(src/cpu/accel.cpp)") if kind == "reference" else "the oracle's SAH BVH"
    return (paths / t_total / 1e6, kind, cores,
            f"{frames} frame(s) of {W}x{rows} at 1 spp ({paths} paths, {t_total:.1f} s); {accel}")


def launch_ranks(n):
    """`bench.py --gpus N` outside torchrun: start N ranks on this node (one
    per GPU) with torch.distributed.run and return its exit status."""
    import socket

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.call(cmd)


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    pt, sc, cam, W, H, spp, depth, cfg = workload(args.workload)
    times = []
    kind = cores = sample = None
    for i in range(args.warmup + args.steps):
        v, kind, cores, sample = cpu_reference_run(pt, sc, cam, W, H, depth, seconds=args.cpu_seconds)
        if i >= args.warmup:
            times.append(v)
    value = float(np.median(times))
    paths_step = W * H * spp
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Mpaths/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": paths_step / (value * 1e6) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(cfg, parallelism="host threads"),
            "cpu_baseline": {"value": value, "unit": "Mpaths/s", "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="pt", choices=["pt", "reference"])
    ap.add_argument("--workload", default="disney_envmap",
                    choices=["disney_envmap", "cornell", "hair_volume", "radiance_cache"])
    ap.add_argument("--env-sampling", default="cdf", choices=["cdf", "alias"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--spp", type=int, default=0, help="override samples per pixel (profiling of small cases)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--wave-paths", type=int, default=0, help="paths in flight per wave (0 = library default)")
    ap.add_argument("--no-ttq", action="store_true", help="skip the time-to-relMSE measurement")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-requests measurement")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip configurations 3 and 5 (reported beside the default workload)")
    ap.add_argument("--media-inline", action="store_true",
                    help="heterogeneous media in the inline form (the reference's draw order) instead of the wavefront")
    ap.add_argument("--cache-kernels-only", action="store_true",
                    help="only the radiance-cache network kernels' roofline (profiling of those kernels)")
    args = ap.parse_args()
    if args.gpus < 1:
        raise SystemExit("--gpus must be >= 1")
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ and args.impl == "pt":
        return launch_ranks(args.gpus)
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.cache_kernels_only:
        pt, sc, cam, W, H, spp, depth, cfg = workload(args.workload)
        ctx = pt.Context(0)
        out = cache_kernel_roofline(pt, ctx)
        ctx.upload(sc)
        out["render_mode"] = cache_render_roofline(pt, ctx, W, H, cam, depth, pt.PT_ENV_CDF)
        print(json.dumps({"cache_roofline": out}), flush=True)
        ctx.close()
        return 0

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        raise SystemExit(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world} ranks were started")
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    pt, sc, cam, W, H, spp, depth, cfg = workload(args.workload)
    if args.spp:
        spp = cfg["spp"] = args.spp
    env_mode = pt.PT_ENV_ALIAS if args.env_sampling == "alias" else pt.PT_ENV_CDF
    ctx = pt.Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    t0 = time.perf_counter()
    ctx.upload(sc)
    upload_s = time.perf_counter() - t0
    D = importlib.import_module("pbrt_b200.distributed")
    film = D.new_film(H, W, device="cuda")  # accumulated frames (sum, Kahan compensation)
    shard = D.new_film(H, W, device="cuda") if world > 1 else None  # this rank's part of a frame
    render_into = D.device_renderer(ctx)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > 126 MB L2
    paths_step = W * H * spp

    base_flags = 0 if args.media_inline else pt.PT_RENDER_MEDIA_WAVEFRONT

    def step(i, timing=False):
        def params(off):
            return pt.render_params(W, H, spp, cam, max_depth=depth, sample_offset=off, env_sampling=env_mode,
                                    wave_paths=args.wave_paths,
                                    flags=base_flags | (pt.PT_RENDER_STAGE_TIMING if timing else 0))

        _, _, st = D.render_frame(render_into, params, film, i, rank, world, spp, shard=shard)
        return st

    def timed_steps(first, timing):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        sts = []
        for k in range(args.steps):
            flush.zero_()
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            ev[k][0].record(stream)
            sts.append(step(first + k, timing=timing))
            ev[k][1].record(stream)
            torch.cuda.synchronize()
        per = [a.elapsed_time(b) for a, b in ev]
        t = sum(per)
        if world > 1:
            tt = torch.tensor([t], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = float(tt.item())
        return t, sts, per

    # the clock sampler starts with the warm-up (its start-up stays out of the
    # timed steps) and keeps sampling through them
    with ClockSampler(local) as clk:
        for i in range(args.warmup):
            step(i)
        torch.cuda.synchronize()
        ms, stats, per_step = timed_steps(args.warmup, timing=False)
    value = paths_step * world * args.steps / (ms / 1e3) / 1e6
    # the same steps again with an event pair around every launch: per-kernel
    # times for the roofline (the headline above carries no per-launch events)
    _, tstats, _ = timed_steps(args.warmup + args.steps, timing=True)

    # end to end through the C ABI with pinned host films (copies in the timed region)
    e2e_value = None
    if not args.no_e2e:
        hsum = torch.zeros((H, W, 4), dtype=torch.float32, pin_memory=True)
        hcomp = torch.zeros_like(hsum, pin_memory=True)
        film_np, comp_np = hsum.numpy(), hcomp.numpy()
        # untimed warm-up through the same call: the library captures its
        # launch graph for the host-film staging buffers on the first call
        for k in range(args.warmup):
            P = pt.render_params(W, H, spp, cam, max_depth=depth, sample_offset=D.sample_offset(k, rank, world, spp),
                                 env_sampling=env_mode, wave_paths=args.wave_paths, flags=base_flags)
            ctx.render(P, film_np, comp_np, pt.PT_MEM_HOST)
        torch.cuda.synchronize()
        e2e_ms = 0.0
        # with several ranks: rank 0 uploads the accumulated host film into its
        # shard, every rank renders its samples, one all-reduce sums the
        # shards and rank 0 downloads the frame (render_frame with host_acc)
        hfilm = torch.stack([hsum, hcomp]).pin_memory() if world > 1 else None
        for k in range(args.steps):
            def e2e_params(off):
                return pt.render_params(W, H, spp, cam, max_depth=depth, sample_offset=off, env_sampling=env_mode,
                                        wave_paths=args.wave_paths, flags=base_flags)
            flush.zero_()
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            if world > 1:
                D.render_frame(render_into, e2e_params, None, k, rank, world, spp, shard=shard, host_acc=hfilm)
            else:
                ctx.render(e2e_params(D.sample_offset(k, rank, world, spp)), film_np, comp_np, pt.PT_MEM_HOST)
            b.record(stream)
            torch.cuda.synchronize()
            e2e_ms += a.elapsed_time(b)
        if world > 1:
            t = torch.tensor([e2e_ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_ms = float(t.item())
        e2e_value = paths_step * world * args.steps / (e2e_ms / 1e3) / 1e6

    ext = sum(s.extension_rays for s in stats)
    sh = sum(s.shadow_rays for s in stats)
    stage_ms = {k: sum(getattr(s, "ms_" + k) for s in tstats)
                for k in ("raygen", "extend", "shade", "shadow", "tail", "film")}
    launches = {"extend": sum(s.bounces for s in tstats)}
    # k_extend's own rays (the tail kernel traces the last bounces' rays itself)
    ext_k = sum(s.extension_rays - s.tail_extension_rays for s in tstats)
    peak, peak_src = measured_peaks()
    dominant = max(stage_ms, key=stage_ms.get)
    # roofline of the closest-hit traversal kernel: algorithmic bytes per launch / mean launch time
    n_ext_launch = max(1, launches["extend"])
    ext_bytes_per_launch = ext_k * BYTES_PER_EXT_RAY / n_ext_launch
    ext_ms_per_launch = stage_ms["extend"] / n_ext_launch
    achieved = ext_bytes_per_launch / (ext_ms_per_launch / 1e3) / 1e9 if ext_ms_per_launch > 0 else 0.0
    traffic = None
    if cfg["workload"] in EXTEND_DRAM_BYTES_PER_RAY:
        traffic = round(EXTEND_DRAM_BYTES_PER_RAY[cfg["workload"]] * ext_k / n_ext_launch, 1)
    n_ext = ext / (paths_step * args.steps)
    n_sh = sh / (paths_step * args.steps)
    b_path = BYTES_PER_PATH_FILM + BYTES_PER_EXT_RAY * n_ext + BYTES_PER_SHADOW_RAY * n_sh
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3),
        "ms_steps": [round(x, 3) for x in per_step], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene, no reference assets)",
        "config": dict(cfg, parallelism=f"sample-range x{world}" if world > 1 else "single GPU",
                       env_sampling=args.env_sampling,
                       l2="flushed between timed steps (256 MiB write); path state > L2"),
        "mrays_per_s": round((ext + sh) * world / (ms / 1e3) / 1e6, 2),
        "per_path": {"extension_rays": round(n_ext, 4), "shadow_rays": round(n_sh, 4),
                     "algorithmic_bytes": round(b_path, 2),
                     "achieved_gbs": round(value * 1e6 * b_path / world / 1e9, 2)},
        "stage_ms_per_step": {k: round(v / args.steps, 3) for k, v in stage_ms.items()},
        "roofline": {"bound": "hbm", "kernel": "k_extend (BVH8 closest hit)", "achieved": round(achieved, 2),
                     "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 5),
                     "traffic": traffic, "peak_source": peak_src,
                     "algorithmic_bytes_per_launch": round(ext_bytes_per_launch, 1),
                     "mean_launch_ms": round(ext_ms_per_launch, 4), "dominant_stage": dominant},
        "e2e": None if e2e_value is None else {
            "value": round(e2e_value, 3), "unit": "Mpaths/s", "h2d_bytes_per_step": 2 * W * H * 16,
            "d2h_bytes_per_step": 2 * W * H * 16,
            "path": "pt_render with pinned host films" if world == 1 else
                    "render_frame: host film -> rank-0 shard, render, NCCL all-reduce, shard -> host film"},
        "gpu_launches": int(sum(s.launches for s in stats)),
        "clocks": clk.summary(),
        "scene_upload_s": round(upload_s, 3),
    }
    if world == 1 and not args.no_ttq:
        line["time_to_relmse"] = time_to_relmse(pt, ctx, stream, W, H, cam, depth, env_mode, max(spp, 64),
                                                calls=CACHE_CALLS.get(cfg["workload"], CACHE_CALLS_DEFAULT))
        line["cache_roofline"] = cache_kernel_roofline(pt, ctx)
        line["cache_roofline"]["render_mode"] = cache_render_roofline(pt, ctx, W, H, cam, depth, env_mode)
    if world == 1 and not args.no_batch:
        line["batched"] = batched_requests_run(pt)
    if world == 1 and not args.no_configs and cfg["workload"] == "disney_envmap":
        # the other single-GPU configurations, each on its own context
        ctx.close()
        ctx = None
        line["config3"] = config3_sweep(pt)
        line["config5"] = config5_run(pt)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, kind, cores, sample = cpu_reference_run(pt, sc, cam, W, H, depth, seconds=args.cpu_seconds)
        line["cpu_baseline"] = {"value": round(v, 4), "unit": "Mpaths/s", "cores": cores, "kind": kind,
                                "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ctx is not None:
        ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
