"""Benchmark: spectral path tracing of the Cornell box workload on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Workload (one "step"): a full 512x512 frame of 256 samples per pixel, 4 hero
wavelengths, maximum path length 8, MIS next-event estimation, FP64 film, on
the seeded procedural Cornell box (vlr_b200.scenes.cornell_box_desc).  Metric:
path segments per second (extension rays traced, camera rays included, each
with its shading and NEE shadow ray), reported in G segments/s.

  value   device-timed throughput of the render call with the scene, film and
          path state resident in HBM (CUDA events, max over ranks);
  e2e     the same metric through the public C API with the step's result
          read back to host memory every step (vlrbContextRenderSamples +
          vlrContextReadOutputBuffer into pinned memory);
  roofline   dominant wavefront stage against the measured HBM bandwidth;
  cpu_baseline  the CPU restatement of the reference path tracer over the
          reference's own BSDF/spectral code, all host threads, bounded sample.

With --gpus N > 1 (under torchrun) every rank renders its own 256 spp of the
same frame (weak scaling) and the FP64 films are summed with one NCCL
all-reduce per step.  --impl reference times the reference's CPU
implementation of the path on the host cores instead.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "time-to-1% RMSE vs FP64 ref, guided vs plain PT on 1 B200; G path segments/s"
UNIT = "G path segments/s"
W = H = 512
SPP_PER_STEP = 256
MAX_PATH_LENGTH = 8


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 8:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[4 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def cpu_baseline(seconds_target=12.0):
    """The reference CPU path: CPU restatement of path_tracing.cu over the
    reference's own BSDF/spectral code (oracle/_ref), all host threads."""
    from oracle import ref
    from vlr_b200 import scenes
    if not ref.available():
        return None
    desc = scenes.cornell_box_desc(W, H)
    flat = scenes.flatten_desc(desc)
    threads = os.cpu_count() or 1
    spp = 1
    states = ref.seed_states(W * H)
    t0 = time.time()
    _, states, seg = ref.pt_render(flat, desc["camera"], W, H, spp, MAX_PATH_LENGTH, rng_states=states,
                                   threads=threads)
    dt = time.time() - t0
    spp = max(1, min(64, int(seconds_target / max(dt, 1e-3))))
    t0 = time.time()
    _, _, seg = ref.pt_render(flat, desc["camera"], W, H, spp, MAX_PATH_LENGTH, rng_states=states,
                              threads=threads)
    dt = time.time() - t0
    return {"value": seg / dt / 1e9, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{W}x{H} Cornell box, {spp} spp, max path length {MAX_PATH_LENGTH} "
                      f"({seg} segments, {dt:.1f} s): CPU restatement of path_tracing.cu over the reference's "
                      f"own BSDF/spectral code, brute-force intersection"}


REFERENCE_ARM_BUDGET_S = 240.0


def run_reference(args):
    """The reference's CPU implementation of the path (the CPU restatement of
    path_tracing.cu over the reference's own BSDF/spectral classes built for
    the host) on all host cores, on this workload: one step = the full
    512x512 frame of 256 spp when warm-up + timed steps fit in about four
    minutes on this host, else as many spp per step as fit (stated in
    config).  Per-pixel RNG seeds are generated once, before any step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference host build oracle/_ref is missing"}))
        return 0
    from vlr_b200 import scenes
    desc = scenes.cornell_box_desc(W, H)
    flat = scenes.flatten_desc(desc)
    threads = os.cpu_count() or 1
    states = ref.seed_states(W * H)
    t0 = time.time()
    _, states, _ = ref.pt_render(flat, desc["camera"], W, H, 1, MAX_PATH_LENGTH, rng_states=states,
                                 threads=threads)
    per_spp = time.time() - t0
    spp_step = SPP_PER_STEP
    if (args.warmup + args.steps) * per_spp * spp_step > REFERENCE_ARM_BUDGET_S:
        spp_step = max(1, int(REFERENCE_ARM_BUDGET_S / ((args.warmup + args.steps) * per_spp)))
    film = np.zeros((H, W, 16), np.float64)
    for _ in range(args.warmup):
        ref.pt_render(flat, desc["camera"], W, H, spp_step, MAX_PATH_LENGTH, rng_states=states, film=film,
                      threads=threads)
    total_seg = 0
    t0 = time.time()
    for _ in range(args.steps):
        film[:] = 0.0
        _, states, seg = ref.pt_render(flat, desc["camera"], W, H, spp_step, MAX_PATH_LENGTH, rng_states=states,
                                       film=film, threads=threads)
        total_seg += seg
    dt = time.time() - t0
    v = total_seg / dt / 1e9
    same = spp_step == SPP_PER_STEP
    workload = (f"Cornell box PT {W}x{H}, {spp_step} spp per step"
                + ("" if same else f" (bounded CPU sample of the {SPP_PER_STEP} spp frame)")
                + f", max path length {MAX_PATH_LENGTH}, 4 hero wavelengths, MIS NEE, FP64 film")
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": workload, "same_spp_as_gpu_arm": same},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{args.steps} steps of {spp_step} spp of {W}x{H}: CPU restatement of "
                                       f"path_tracing.cu over the reference's own BSDF/spectral code built for the "
                                       f"host, OpenMP over rows, brute-force intersection"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---- time to 1% error, guided vs plain path tracing (glossy-caustic scene)
RMSE_W = RMSE_H = 1024
RMSE_BLOCK = 8
RMSE_TARGET = 0.01
RMSE_REF_SPP = 16384
RMSE_CHUNK_SPP = 16
RMSE_CAP_S = 40.0
RMSE_PIXEL_TARGET = 0.10


class _FilmView:
    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "version": 3, "data": (ptr, False)}


def _cmf_y():
    import ctypes
    from vlr_b200 import lib
    L = lib()
    L.vlrbCmfStrata.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    xyz = np.zeros(48, np.float32)
    integ = ctypes.c_float()
    L.vlrbCmfStrata(xyz.ctypes.data_as(ctypes.c_void_p), ctypes.byref(integ))
    return xyz[16:32].astype(np.float64)


def time_to_rmse():
    """Device time until the image is within RMSE_TARGET of an FP64 plain-PT
    reference (RMSE_REF_SPP spp in two independently seeded halves), for
    plain and for guided path tracing with online training included in the
    time.  Error: RMSE of RMSE_BLOCK^2-pixel block means of CIE Y, relative
    to the reference mean; beside it the per-pixel relative RMSE of CIE Y at
    every checkpoint and the time to RMSE_PIXEL_TARGET per pixel (a per-pixel
    1% needs far more samples than either method renders in the cap).  The
    reference's own variance, a quarter of the halves' mean squared
    difference, is subtracted from every squared error, per block and per
    pixel.  A method that has not reached a target after RMSE_CAP_S seconds
    reports its error there and an extrapolated time assuming error ~
    1/sqrt(time)."""
    import torch
    from vlr_b200 import vlr as V, scenes
    W, H, b = RMSE_W, RMSE_H, RMSE_BLOCK
    cy = torch.tensor(_cmf_y(), device="cuda")

    def make(guided, seed):
        ctx = V.Context()
        ctx.bindOutputBuffer(W, H)
        scene, cam, keep = scenes.cornell_box(ctx, W, H, glass="sphere", light_scale=0.1)
        ctx.setScene(scene)
        ctx.setOptions(max_path_length=MAX_PATH_LENGTH, max_paths_in_flight=1 << 24, rng_seed=seed,
                       consistent_dielectric_pdf=True)
        if guided:
            # guided and trained at the first bounce; after one warm-up
            # launch (16 spp) one training step every 4 launches (64 spp: the
            # fastest of the measured schedules, 1-2 guided bounces x a step
            # every 4-64 spp)
            ctx.setGuiding(enabled=True, train=True, recordBounces=1, warmupLaunches=1, trainInterval=4)
        return ctx, cam, keep

    def pixels(ctx):
        f = torch.as_tensor(_FilmView(ctx.film_device_ptr(), W * H * 16), device="cuda").view(H, W, 16)
        return f @ cy

    def blocks(y):
        return y.view(H // b, b, W // b, b).mean(dim=(1, 3))

    # the reference in two independent halves: their difference measures the
    # reference's own noise, which is subtracted from every squared error
    halves = []
    for seed in (0x9E3779B97F4A7C15, 0xD1B54A32D192ED03):
        ctx, cam, keep = make(False, seed)
        for k in range(RMSE_REF_SPP // 2 // 1024):
            ctx.render_samples(cam, k == 0, 1024)
        halves.append(pixels(ctx) / (RMSE_REF_SPP // 2))
        torch.cuda.synchronize()
        ctx.close()
    ref_px = 0.5 * (halves[0] + halves[1])
    ref_var_px = (torch.mean((halves[0] - halves[1]) ** 2) / 4).item()
    ref = blocks(ref_px)
    ref_var = (torch.mean((blocks(halves[0]) - blocks(halves[1])) ** 2) / 4).item()
    ref_mean = ref.mean().item()
    out = {"scene": "Cornell box, 20,022-triangle GGX dielectric sphere (IOR 1.5, roughness 0.02), light 0.1x area",
           "resolution": [W, H], "max_path_length": MAX_PATH_LENGTH, "target": RMSE_TARGET,
           "error": f"RMSE of {b}x{b}-pixel block means of CIE Y / reference mean",
           "pixel_error": "RMSE of per-pixel CIE Y / reference mean (curve entries' fourth value)",
           "pixel_target": RMSE_PIXEL_TARGET,
           "reference": f"plain PT, {RMSE_REF_SPP} spp in two independently seeded halves, FP64 film; "
                        f"the reference's own variance (a quarter of the halves' mean squared difference) is "
                        f"subtracted from each squared error",
           "reference_noise": None,
           "reference_pixel_noise": None,
           "dielectric_pdf": "consistent (the reference's MicrofacetScattering pdf is 0 for exits: "
                             "NEE double counting and fireflies)",
           "guided_config": "hash grid 16x2x2^19, 3x64 BF16 MLP, 8 vMF lobes, Adam lr 1e-2, 2^18 samples per "
                            "step, one-sample MIS 0.5 with the BSDF; guided and trained at the first bounce, "
                            "one warm-up launch of 16 spp, then one step every 4 launches (64 spp); training time "
                            "included"}
    out["reference_noise"] = math.sqrt(ref_var) / ref_mean
    out["reference_pixel_noise"] = math.sqrt(ref_var_px) / ref_mean
    for name, guided in (("plain", False), ("guided", True)):
        ctx, cam, keep = make(guided, 0)
        stream = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t = 0.0
        n = 0
        curve = []
        reached = None
        pixel_reached = None
        while t < RMSE_CAP_S:
            e0.record(stream)
            ctx.render_samples(cam, n == 0, RMSE_CHUNK_SPP, stream=stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            t += e0.elapsed_time(e1) * 1e-3
            n += RMSE_CHUNK_SPP
            y = pixels(ctx) / n
            mse = torch.mean((blocks(y) - ref) ** 2).item()
            err = math.sqrt(max(mse - ref_var, 0.0)) / ref_mean
            mse_px = torch.mean((y - ref_px) ** 2).item()
            err_px = math.sqrt(max(mse_px - ref_var_px, 0.0)) / ref_mean
            if pixel_reached is None and err_px <= RMSE_PIXEL_TARGET:
                pixel_reached = t
            if n in (16, 64, 256, 1024, 4096, 8192) or err <= RMSE_TARGET:
                curve.append([n, round(t, 4), err, err_px])
            if err <= RMSE_TARGET:
                reached = t
                break
        r = {"seconds": reached, "spp": n, "error_at_end": err, "pixel_error_at_end": err_px,
             "seconds_at_end": t, "seconds_to_pixel_target": pixel_reached, "curve": curve}
        if reached is None:
            r["seconds_extrapolated"] = t * (err / RMSE_TARGET) ** 2
        if pixel_reached is None:
            r["seconds_to_pixel_target_extrapolated"] = t * (err_px / RMSE_PIXEL_TARGET) ** 2
        if guided:
            r["guiding"] = ctx.guiding_stats()
        seg = ctx.stats()["pathSegments"]
        r["segments_per_s"] = seg / t / 1e9
        out[name] = r
        ctx.close()
    tp = out["plain"]["seconds"] or out["plain"]["seconds_extrapolated"]
    tg = out["guided"]["seconds"] or out["guided"]["seconds_extrapolated"]
    out["guided_over_plain"] = tg / tp
    pp = out["plain"]["seconds_to_pixel_target"] or out["plain"]["seconds_to_pixel_target_extrapolated"]
    pg = out["guided"]["seconds_to_pixel_target"] or out["guided"]["seconds_to_pixel_target_extrapolated"]
    out["guided_over_plain_pixel"] = pg / pp
    return out


# ---- the other scope-table workloads, reported beside the headline line
BATCH_BYTES_PER_QUERY = 116     # in: wo 12, material 4, roughness 8, ior 4, albedo 12, metallic 4, u 12,
                                # wavelength u 8; out: value 16, pdf 4, wi 12, eval value 16, eval pdf 4
# ncu, one launch of the 2^20-query batch (--set full): DRAM bytes read +
# written, FMA-pipe and issue-active fractions; the kernel is issue/latency
# bound inside the GGX BSDFs, so these stand beside its HBM fraction.
BATCH_NCU = {"dram_bytes": 177.8e6 + 93.7e6, "fma_pipe": 0.243, "issue": 0.480}


def bsdf_batch_workload(hbm_peak):
    """2^20-query BSDF shading batches (device-resident SoA, 8 distinct
    batches rotated so the 0.97 GB working set exceeds L2), CUDA-event
    timed; the CPU leg is the reference's BSDF classes built for the host on
    all cores over a bounded sample."""
    import torch
    import vlr_b200 as VB
    n = 1 << 20
    dev = torch.device("cuda")
    batches = []
    for b in range(8):
        inp = VB.make_bsdf_batch_inputs(n, seed=100 + b)
        din = {k: torch.from_numpy(np.ascontiguousarray(inp[k])).to(dev) for k in VB.BATCH_INPUTS}
        dout = {k: torch.empty((n, c) if c > 1 else n, dtype=torch.float32, device=dev)
                for k, c in VB.BATCH_OUTPUTS.items()}
        batches.append((din, dout))
    stream = torch.cuda.current_stream()
    for i in range(8):
        VB.bsdf_batch_device(*batches[i % 8], stream.cuda_stream)
    iters = 64
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for i in range(iters):
        VB.bsdf_batch_device(*batches[i % 8], stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / iters
    gbs = n * BATCH_BYTES_PER_QUERY / (ms * 1e-3) / 1e9
    # end to end through the host-buffer entry (vlrbBsdfBatchHost: device
    # buffers, H2D copy of the inputs, the kernel, D2H copy of the outputs),
    # host-clock timed since the call returns when its results are home
    src = VB.make_bsdf_batch_inputs(n, seed=100)
    host_inp = {}
    for k in VB.BATCH_INPUTS:      # pinned host arrays, as a caller streaming batches would keep them
        a = np.ascontiguousarray(src[k])
        t = torch.empty(a.shape, dtype=getattr(torch, a.dtype.name), pin_memory=True)
        t.numpy()[...] = a
        host_inp[k] = t.numpy()
    host_out = {k: torch.empty((n, c) if c > 1 else (n,), dtype=torch.float32, pin_memory=True).numpy()
                for k, c in VB.BATCH_OUTPUTS.items()}
    VB.bsdf_batch_host(host_inp, outputs=host_out)
    reps = 16
    t0 = time.perf_counter()
    for _ in range(reps):
        VB.bsdf_batch_host(host_inp, outputs=host_out)
    e2e_s = (time.perf_counter() - t0) / reps
    out = {"workload": "BSDF shading batch, 2^20 queries, seven BSDFs uniform, 4 hero wavelengths",
           "queries_per_s": n / (ms * 1e-3), "ms_per_batch": ms,
           "e2e": {"value": n / e2e_s, "unit": "queries/s", "h2d_bytes_per_step": n * 64, "d2h_bytes_per_step": n * 52,
                   "note": "vlrbBsdfBatchHost between pinned host arrays, host-clock timed"},
           "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm_peak, "unit": "GB/s", "frac": gbs / hbm_peak,
                        "bytes_per_query": BATCH_BYTES_PER_QUERY,
                        "fp32_pipe_active": BATCH_NCU["fma_pipe"], "issue_active": BATCH_NCU["issue"],
                        "traffic": BATCH_NCU["dram_bytes"],
                        "ncu_source": "dram__bytes_read.sum + dram__bytes_write.sum, FMA pipe and issue-active "
                                      "fractions of one launch of this workload"}}
    from oracle import ref
    if ref.available():
        m = 1 << 16
        inp = VB.make_bsdf_batch_inputs(m, seed=7)
        threads = os.cpu_count() or 1
        t0 = time.time()
        reps = 0
        while time.time() - t0 < 3.0:
            ref.bsdf_batch(inp, threads=threads)
            reps += 1
        dt = time.time() - t0
        out["cpu_baseline"] = {"value": reps * m / dt, "unit": "queries/s", "cores": threads, "kind": "reference",
                               "sample": f"{reps} x 2^16 queries: the reference's BSDF classes (materials.cu) "
                                         f"built for the host, OpenMP"}
    return out


TERRAIN_CPU_W, TERRAIN_CPU_H = 192, 108


def terrain_cpu_baseline(desc, renderer, seconds_target=10.0):
    """The reference's CPU implementation of the terrain workload's
    integrator (CPU restatements of path_tracing.cu / lvc_bpt.cu over the
    reference's BSDF/spectral classes, the environment light with the
    reference's own importance map, a median-split BVH over the same 3.4 M
    triangles), all host threads, at 1/10 of the resolution; timed over the
    render loops only (scene and hierarchy set-up excluded, as on the GPU)."""
    from oracle import ref
    from vlr_b200 import scenes
    if not ref.available():
        return None
    W, H = TERRAIN_CPU_W, TERRAIN_CPU_H
    flat = scenes.flatten_instanced_desc(desc)
    cam = dict(desc["camera"])
    cam["aspect"] = W / H
    threads = os.cpu_count() or 1
    ref.env_set(desc["env"], mode=1)
    try:
        def run(spp):
            if renderer == "pt":
                _, _, seg = ref.pt_render(flat, cam, W, H, spp, 12, threads=threads)
            else:
                _, _, seg, _ = ref.bpt_render(flat, cam, W, H, spp, 12, W * H, threads=threads)
            return seg, ref.last_render_seconds()
        seg, dt = run(1)
        spp = max(1, min(256, int(seconds_target / max(dt, 1e-3))))
        seg, dt = run(spp)
    finally:
        ref.env_set(None)
    name = "path_tracing.cu" if renderer == "pt" else "lvc_bpt.cu (one light subpath per pixel per frame)"
    return {"value": seg / dt / 1e9, "unit": "G path segments/s", "cores": threads, "kind": "port",
            "sample": f"{W}x{H} (1/10 of the 1920x1080 frame), {spp} spp, max depth 12, {len(flat['tris'])} "
                      f"triangles ({seg} segments in {dt:.1f} s): CPU restatement of {name} over the reference's "
                      f"own BSDF/spectral code"}


def terrain_workloads(names=("terrain_pt", "terrain_lvc_bpt"), cpu=True, paths_in_flight=0):
    """Path tracing and LVC-BPT on the 2,097,152-triangle terrain with 4096
    instanced icospheres under the 2048x1024 sky (FP64 CDF), 1920x1080,
    max depth 12, one light subpath per pixel per frame for LVC-BPT;
    device-timed segments/s after warm-up (8 and 4 spp: bounded samples of
    the 64-spp frame), the dominant wavefront stage against the HBM
    roofline, and the CPU restatement on the host cores beside it.
    paths_in_flight > 0 fixes the launch size instead of autotuning it (a
    smaller device footprint, for profiling)."""
    import torch
    from vlr_b200 import vlr as V, scenes
    W, H = 1920, 1080
    desc = scenes.terrain_scene_desc(W, H)
    hbm_peak, peak_kind = measured_peaks()
    out = {}
    for name, renderer, spp in (("terrain_pt", V.RENDERER_PATH_TRACING, 8), ("terrain_lvc_bpt", V.RENDERER_BPT, 4)):
        if name not in names:
            continue
        ctx = V.Context()
        ctx.bindOutputBuffer(W, H)
        scene, cam, keep = scenes.build_instanced(ctx, desc)
        ctx.setScene(scene)
        ctx.setRenderer(renderer)
        ctx.setOptions(max_path_length=12, max_paths_in_flight=1 << 22)
        if paths_in_flight:
            ctx.setOptions(max_paths_in_flight=paths_in_flight)
        elif renderer == V.RENDERER_PATH_TRACING:
            ctx.autotune(cam, spp)      # launch configuration for this workload's frame
        ctx.render_samples(cam, True, 2)
        torch.cuda.synchronize()
        s0 = ctx.stats()["pathSegments"]
        stream = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.render_samples(cam, False, spp, stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        seg = ctx.stats()["pathSegments"] - s0
        st = ctx.stats()
        # per-stage device times of one more call of the same size (stage
        # events serialise the stages a little: they sum to slightly more than
        # the timed call), reported per spp
        ctx.set_profiling(True)
        ctx.kernel_times(reset=True)
        q0 = ctx.stats()
        ctx.render_samples(cam, False, spp, stream=stream.cuda_stream)
        torch.cuda.synchronize()
        stages, _ = ctx.kernel_times(reset=True)
        q1 = ctx.stats()
        ctx.set_profiling(False)
        rays = q1["pathSegments"] - q0["pathSegments"]
        r = {"workload": f"{'path tracing' if renderer == V.RENDERER_PATH_TRACING else 'LVC-BPT'} "
                         f"{W}x{H}, {spp} spp per timed call (bounded sample of the 64-spp frame), max depth 12, "
                         f"sky with sun (FP64 CDF)",
             "triangles": st["numTriangles"], "segments_per_s": seg / (ms * 1e-3) / 1e9,
             "unit": "G path segments/s", "ms": ms,
             "stage_ms_per_spp": {k: v["ms"] / spp for k, v in stages.items() if v["ms"] > 0}}
        if renderer == V.RENDERER_PATH_TRACING:
            dom = max(("trace", "shade", "shadow"), key=lambda k: stages[k]["ms"])
            units = rays if dom != "shadow" else q1["shadowRays"] - q0["shadowRays"]
            gbs = STAGE_BYTES[dom] * units / (stages[dom]["ms"] * 1e-3) / 1e9
            r["roofline"] = {"bound": "hbm", "kernel": dom + "Kernel", "achieved": gbs, "peak": hbm_peak,
                             "unit": "GB/s", "frac": gbs / hbm_peak, "peak_source": peak_kind,
                             "bytes_per_unit": STAGE_BYTES[dom],
                             "note": "algorithmic bytes of the wavefront state; BVH node traffic excluded"}
        else:
            r["light_vertex_overflow"] = st["lightVertexOverflow"]
        if cpu:
            try:
                r["cpu_baseline"] = terrain_cpu_baseline(desc, "pt" if renderer == V.RENDERER_PATH_TRACING else "bpt")
            except Exception as ex:  # reported, never fatal for the GPU line
                r["cpu_baseline"] = {"error": str(ex)}
        out[name] = r
        ctx.close()
    return out


def glossy_guided_workload():
    """Guided path tracing with online training on the Cornell box with the
    20,022-triangle GGX dielectric sphere and the light at 0.1x area,
    1024x1024, max path length 8, consistent dielectric pdf: 16 spp of
    warm-up training, then 16 spp in 4 launches timed per stage (the
    workload of the guiding-kernel profiles)."""
    import torch
    from vlr_b200 import vlr as V, scenes
    W = H = 1024
    ctx = V.Context()
    ctx.bindOutputBuffer(W, H)
    scene, cam, keep = scenes.cornell_box(ctx, W, H, glass="sphere", light_scale=0.1)
    ctx.setScene(scene)
    ctx.setOptions(max_path_length=8, max_paths_in_flight=1 << 22, consistent_dielectric_pdf=True)
    ctx.setGuiding(enabled=True, train=True)
    ctx.render_samples(cam, True, 16)
    torch.cuda.synchronize()
    ctx.set_profiling(True)
    ctx.kernel_times(reset=True)
    s0 = ctx.stats()
    ctx.render_samples(cam, False, 16)
    torch.cuda.synchronize()
    stages, _ = ctx.kernel_times(reset=True)
    s1 = ctx.stats()
    ctx.set_profiling(False)
    seg = s1["pathSegments"] - s0["pathSegments"]
    total_ms = sum(v["ms"] for v in stages.values())
    out = {"workload": "guided PT with online training, Cornell box with GGX dielectric sphere, light 0.1x, "
                       "1024x1024, 16 spp, max path length 8",
           "segments_per_s": seg / (total_ms * 1e-3) / 1e9, "unit": "G path segments/s",
           "stage_ms": {k: v["ms"] for k, v in stages.items()}, "guiding": ctx.guiding_stats()}
    ctx.close()
    return out


def light_tracing_workload(cpu=True):
    """The light tracer (light subpaths with lens connections splatted to the
    film) on the Cornell box workload's scene, 512x512, one light subpath per
    pixel per frame, 64 frames in one launch of 2^24 light subpaths, max path
    length 8; device-timed segments/s."""
    import torch
    from vlr_b200 import vlr as V, scenes
    ctx = V.Context()
    ctx.bindOutputBuffer(W, H)
    scene, cam, keep = scenes.build(ctx, scenes.cornell_box_desc(W, H))
    ctx.setScene(scene)
    ctx.setRenderer(V.RENDERER_LIGHT_TRACING)
    ctx.setOptions(max_path_length=MAX_PATH_LENGTH, max_paths_in_flight=1 << 24)     # 64 frames per launch
    stream = torch.cuda.current_stream()
    ctx.render_samples(cam, True, 64, stream=stream.cuda_stream)     # warm-up: buffers sized and seeded
    torch.cuda.synchronize()
    s0 = ctx.stats()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.render_samples(cam, False, 64, stream=stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    s1 = ctx.stats()
    out = {"workload": f"light tracing, Cornell box {W}x{H}, {W * H} light subpaths per frame, 64 frames in "
                       f"one launch, max path length {MAX_PATH_LENGTH}",
           "segments_per_s": (s1["pathSegments"] - s0["pathSegments"]) / (ms * 1e-3) / 1e9,
           "lens_connections_per_s": (s1["shadowRays"] - s0["shadowRays"]) / (ms * 1e-3) / 1e9,
           "unit": "G path segments/s", "ms": ms}
    ctx.close()
    if cpu:
        # the CPU restatement of light_tracing.cu, all host threads, on a
        # bounded sample of the same workload (4 frames)
        from oracle import ref
        if ref.available():
            desc = scenes.cornell_box_desc(W, H)
            frames = 4
            _, _, seg = ref.lt_render(scenes.flatten_desc(desc), desc["camera"], W, H, frames, MAX_PATH_LENGTH, W * H)
            secs = ref.last_render_seconds()
            out["cpu_baseline"] = {"value": seg / secs / 1e9, "unit": "G path segments/s",
                                   "cores": os.cpu_count() or 1, "kind": "port",
                                   "sample": f"{frames} frames of {W * H} light subpaths: CPU restatement of "
                                             "light_tracing.cu over the reference's BSDF/spectral code"}
    return out


def denoise_workload():
    """vlrContextRender at 1920x1080 on the Cornell box, one sample per call,
    without and with denoise: the difference per call is the post-processing
    (guide sample: a camera ray, hit decode and base colour per pixel; guide
    conversion; demodulation, five a-trous passes, remodulation).
    Device-timed with CUDA events over 16 calls each."""
    import torch
    from vlr_b200 import vlr as V, scenes
    w, h, calls = 1920, 1080, 16
    ctx = V.Context()
    ctx.bindOutputBuffer(w, h)
    scene, cam, keep = scenes.build(ctx, scenes.cornell_box_desc(w, h))
    ctx.setScene(scene)
    ctx.setOptions(max_path_length=MAX_PATH_LENGTH)
    stream = torch.cuda.current_stream()
    times = {}
    for denoise in (False, True, False, True):      # the first pair warms up
        ctx.render(cam, True, stream=stream.cuda_stream, denoise=denoise)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(calls):
            ctx.render(cam, False, stream=stream.cuda_stream, denoise=denoise)
        e1.record(stream)
        torch.cuda.synchronize()
        times[denoise] = e0.elapsed_time(e1) / calls
    ctx.close()
    post = times[True] - times[False]
    return {"workload": f"denoise: Cornell box {w}x{h}, vlrContextRender 1 spp per call, max path length "
                        f"{MAX_PATH_LENGTH}, with and without denoise = true",
            "render_ms_per_call": times[False], "render_and_denoise_ms_per_call": times[True],
            "post_ms_per_call": post, "post_mpixels_per_s": w * h / (post * 1e-3) / 1e6 if post > 0 else None}


WORKLOADS = {
    "bsdf_batch": lambda a: {"bsdf_batch": bsdf_batch_workload(measured_peaks()[0])},
    "terrain_pt": lambda a: terrain_workloads(("terrain_pt",), cpu=not a.no_cpu_baseline,
                                              paths_in_flight=a.paths_in_flight),
    "terrain_lvc_bpt": lambda a: terrain_workloads(("terrain_lvc_bpt",), cpu=not a.no_cpu_baseline,
                                                   paths_in_flight=a.paths_in_flight),
    "multi_scene_batch": lambda a: {"multi_scene_batch": batch_workload()},
    "glossy_guided": lambda a: {"glossy_guided": glossy_guided_workload()},
    "light_tracing": lambda a: {"light_tracing": light_tracing_workload(cpu=not a.no_cpu_baseline)},
    "denoise": lambda a: {"denoise": denoise_workload()},
    "time_to_rmse": lambda a: {"time_to_rmse": time_to_rmse()},
}


def batch_workload():
    """32 seeded scenes of uneven size (triangles log-uniform in [1k, 2M]
    from the terrain/instance generator; resolution from {256^2, 512^2,
    1024x768, 1920x1080}; 1-64 spp; odd scenes guided with online training),
    each context's paths in flight and blocks per SM chosen by the
    autotuner.  Rendered once as plain per-scene launches one after another,
    then as one CUDA graph of all scenes replayed (vlrbRenderBatch*), then
    as one graph whose plain scenes render in a single persistent kernel
    launch beside the guided scenes' launches (VLRB_BATCH_PERSISTENT);
    reports aggregate segments/s and per-scene frame latency p50/p99 for
    each."""
    import torch
    from vlr_b200 import vlr as V, scenes
    rng = np.random.default_rng(2024)
    resolutions = [(256, 256), (512, 512), (1024, 768), (1920, 1080)]
    items = []
    for k in range(32):
        tris = float(np.exp(rng.uniform(np.log(1e3), np.log(2e6))))
        n_spheres = max(1, int(0.3 * tris / 320))
        cells = max(8, int(np.sqrt(0.7 * tris / 2)))
        W, H = resolutions[int(rng.integers(0, 4))]
        spp = int(np.exp(rng.uniform(0, np.log(64))))
        desc = scenes.terrain_scene_desc(W, H, cells=cells, n_spheres=n_spheres, seed=100 + k, sky=(256, 128))
        ctx = V.Context()
        ctx.bindOutputBuffer(W, H)
        scene, cam, keep = scenes.build_instanced(ctx, desc)
        ctx.setScene(scene)
        ctx.setOptions(max_path_length=8, max_paths_in_flight=min(1 << 22, W * H * spp))
        if k % 2 == 1:
            ctx.setGuiding(enabled=True, train=True, log2TableSize=16, samplesPerStep=1 << 16)
        items.append((ctx, cam, keep, spp, W, H))
    for ctx, cam, keep, spp, W, H in items:
        ctx.autotune(cam, samples_per_trial=min(spp, 4))
    stream = torch.cuda.current_stream()
    ev = lambda: torch.cuda.Event(enable_timing=True)
    # per-scene launches, one scene after another (after one warm-up pass)
    for ctx, cam, keep, spp, W, H in items:
        ctx.render_samples(cam, True, spp, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    seg0 = sum(c.stats()["pathSegments"] for c, *_ in items)
    lat = []
    t0 = ev()
    t0.record(stream)
    for ctx, cam, keep, spp, W, H in items:
        a, b = ev(), ev()
        a.record(stream)
        ctx.render_samples(cam, True, spp, stream=stream.cuda_stream)
        b.record(stream)
        lat.append((a, b))
    t1 = ev()
    t1.record(stream)
    torch.cuda.synchronize()
    seq_ms = t0.elapsed_time(t1)
    seq_lat = [a.elapsed_time(b) for a, b in lat]
    seq_seg = sum(c.stats()["pathSegments"] for c, *_ in items) - seg0
    # one graph of all scenes
    batch = V.RenderBatch([(ctx, cam, spp, True) for ctx, cam, keep, spp, W, H in items])
    batch.launch(stream.cuda_stream)
    torch.cuda.synchronize()
    reps = 3
    seg0 = sum(c.stats()["pathSegments"] for c, *_ in items)
    g_lat = []
    t0 = ev()
    t0.record(stream)
    for _ in range(reps):
        batch.launch(stream.cuda_stream)
        g_lat += batch.item_times()
    t1 = ev()
    t1.record(stream)
    torch.cuda.synchronize()
    g_ms = t0.elapsed_time(t1) / reps
    g_seg = (sum(c.stats()["pathSegments"] for c, *_ in items) - seg0) / reps
    batch.close()
    # one graph: the plain scenes in one persistent kernel launch
    pbatch = V.RenderBatch([(ctx, cam, spp, True) for ctx, cam, keep, spp, W, H in items], persistent=True)
    pbatch.launch(stream.cuda_stream)
    torch.cuda.synchronize()
    seg0 = sum(c.stats()["pathSegments"] for c, *_ in items)
    p_lat, p_lat_plain = [], []
    t0 = ev()
    t0.record(stream)
    for _ in range(reps):
        pbatch.launch(stream.cuda_stream)
        times = pbatch.item_times()
        p_lat += times
        p_lat_plain += [t for k, t in enumerate(times) if k % 2 == 0]
    t1 = ev()
    t1.record(stream)
    torch.cuda.synchronize()
    p_ms = t0.elapsed_time(t1) / reps
    p_seg = (sum(c.stats()["pathSegments"] for c, *_ in items) - seg0) / reps
    pbatch.close()
    out = {"workload": "32 seeded terrain/instance scenes, 1k-2M triangles (log-uniform), 256^2..1920x1080, "
                       "1-64 spp, half guided, autotuned launch configuration",
           "triangles": [int(c.stats()["numTriangles"]) for c, *_ in items],
           "per_scene_launches": {"segments_per_s": seq_seg / (seq_ms * 1e-3) / 1e9, "ms": seq_ms,
                                  "latency_ms_p50": float(np.percentile(seq_lat, 50)),
                                  "latency_ms_p99": float(np.percentile(seq_lat, 99))},
           "graph_batch": {"segments_per_s": g_seg / (g_ms * 1e-3) / 1e9, "ms": g_ms,
                           "latency_ms_p50": float(np.percentile(g_lat, 50)),
                           "latency_ms_p99": float(np.percentile(g_lat, 99))},
           "persistent_batch": {"segments_per_s": p_seg / (p_ms * 1e-3) / 1e9, "ms": p_ms,
                                "latency_ms_p50": float(np.percentile(p_lat, 50)),
                                "latency_ms_p99": float(np.percentile(p_lat, 99)),
                                "plain_latency_ms_p50": float(np.percentile(p_lat_plain, 50)),
                                "plain_latency_ms_p99": float(np.percentile(p_lat_plain, 99)),
                                "note": "16 plain scenes in one persistent kernel launch (pixels from one "
                                        "counter, smallest work first), 16 guided scenes as their own launch "
                                        "sequences beside it, all in one replayed CUDA graph"},
           "unit": "G path segments/s"}
    for ctx, *_ in items:
        ctx.close()
    return out


# Algorithmic bytes per unit of work of each wavefront stage (SoA path state,
# counted once per read or write; BVH traffic excluded):
#   trace: queue index 4 + ray 32 + hit 16 + bucket append 4          = 56 B / ray
#   shade: bucket index 4 + flags 4 + wavelengths 16 + hit 16 + ray 32
#          + throughput 16x2 + contribution 16x2 + rng 8x2 + pdf/type 8x2
#          + triangle gather 3x48 (pos/nrm/tan) + index 16 + next ray 32
#          + next-queue append 4 + shadow ray 48                      = 412 B / hit
#   shadow: shadow ray 48 + contribution read-modify-write 32        = 80 B / shadow ray
STAGE_BYTES = {"trace": 56, "shade": 412, "shadow": 80}
# DRAM bytes per path segment of each stage: dram__bytes_read.sum +
# dram__bytes_write.sum over the 8 bounces of one launch of this workload at
# 2^22 paths in flight (ncu, one pass), divided by that launch's segments
# (one sixteenth of a 256-spp step); the bench's own launches (2^25 paths)
# keep less path state in L2 and measured 1.19x these figures.
STAGE_DRAM_BYTES_PER_SEGMENT = {"trace": 69.0, "shade": 357.7, "shadow": 38.2}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="vlr_b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-rmse", action="store_true", help="skip the time-to-1%%-error measurement")
    ap.add_argument("--no-workloads", action="store_true", help="skip the BSDF-batch and terrain workloads")
    ap.add_argument("--paths-in-flight", type=int, default=0,
                    help="pin the launch configuration instead of autotuning it (profiling runs)")
    ap.add_argument("--blocks-per-sm", type=int, default=0)
    ap.add_argument("--workload", choices=sorted(WORKLOADS),
                    help="run only this secondary workload and print its JSON line (profiling runs)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload:
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        print(json.dumps(WORKLOADS[args.workload](args)), flush=True)
        return

    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    from vlr_b200 import vlr as V, scenes

    ctx = V.Context()
    ctx.bindOutputBuffer(W, H)
    desc = scenes.cornell_box_desc(W, H)
    scene, cam, keep = scenes.build(ctx, desc)
    ctx.setScene(scene)
    ctx.setOptions(max_path_length=MAX_PATH_LENGTH, max_paths_in_flight=1 << 22)
    if world > 1:
        # every rank its own sample streams (rank 0 keeps the reference's seed)
        from vlr_b200 import multigpu
        ctx.setOptions(rng_seed=multigpu.rank_seed(rank))
    stream = torch.cuda.current_stream().cuda_stream
    # launch configuration (paths in flight x blocks per SM) chosen by the
    # library's autotuner, one full step per candidate, before any timing
    if args.paths_in_flight:
        ctx.setOptions(max_paths_in_flight=args.paths_in_flight, blocks_per_sm=args.blocks_per_sm or 8)
        chosen = "pinned on the command line"
    else:
        ctx.autotune(cam, SPP_PER_STEP, stream=stream)
        chosen = "vlrbContextAutotune, 2^20..2^25 paths x 4..32 blocks per SM, one step per candidate"
    launch_opts = ctx.options()

    film_t = None
    if world > 1:
        from vlr_b200 import multigpu
        film_t = multigpu.film_tensor(ctx)

    def step():
        ctx.render_samples(cam, True, SPP_PER_STEP, stream=stream)
        if film_t is not None:
            multigpu.allreduce_film(film_t)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    seg0 = ctx.stats()["pathSegments"]
    ctx.kernel_times(reset=True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    seg = ctx.stats()["pathSegments"] - seg0
    _, launches = ctx.kernel_times()
    param_bytes = ctx.launch_param_bytes()
    if world > 1:
        ms_max, seg_total = multigpu.combine(ms, seg)
    else:
        ms_max, seg_total = ms, float(seg)
    value = seg_total / (ms_max * 1e-3) / 1e9

    # ---- end to end through the C API, result read back to pinned host memory
    out_host = torch.empty((H, W, 4), dtype=torch.float32).pin_memory()
    out_np = out_host.numpy()
    seg1 = ctx.stats()["pathSegments"]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
        ctx.read_output(out_np)
    t_e2e = time.perf_counter() - t0
    seg_e2e = ctx.stats()["pathSegments"] - seg1
    if world > 1:
        t_e2e, seg_e2e = multigpu.combine(t_e2e, seg_e2e)
    e2e = seg_e2e / t_e2e / 1e9

    # ---- per-stage device times (separate profiled pass; events add syncs)
    ctx.set_profiling(True)
    ctx.kernel_times(reset=True)
    q0 = ctx.stats()
    for _ in range(2):
        step()
    torch.cuda.synchronize()
    stages, _ = ctx.kernel_times(reset=True)
    q1 = ctx.stats()
    ctx.set_profiling(False)
    rays = q1["pathSegments"] - q0["pathSegments"]
    shadow = q1["shadowRays"] - q0["shadowRays"]
    units = {"trace": rays, "shade": rays, "shadow": shadow}
    hbm_peak, peak_kind = measured_peaks()
    dominant = max(("trace", "shade", "shadow"), key=lambda k: stages[k]["ms"])
    st = stages[dominant]
    per_launch_ms = st["ms"] / max(st["launches"], 1)
    bytes_per_launch = STAGE_BYTES[dominant] * units[dominant] / max(st["launches"], 1)
    achieved = bytes_per_launch / (per_launch_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": dominant + "Kernel", "achieved": achieved, "peak": hbm_peak,
                "unit": "GB/s", "frac": achieved / hbm_peak, "traffic": None,
                "peak_source": peak_kind,
                "stage_ms_per_step": {k: v["ms"] / 2 for k, v in stages.items()}}
    roofline["traffic"] = STAGE_DRAM_BYTES_PER_SEGMENT[dominant] * rays / max(st["launches"], 1)
    roofline["traffic_source"] = ("ncu dram__bytes_read.sum + dram__bytes_write.sum per segment of this workload "
                                  "captured at 2^22 paths in flight, scaled by this launch's segments")

    workloads = None
    if rank == 0 and world == 1 and not args.no_workloads:
        workloads = {}
        for fn in (lambda: {"bsdf_batch": bsdf_batch_workload(hbm_peak)}, terrain_workloads,
                   lambda: {"multi_scene_batch": batch_workload()},
                   lambda: {"light_tracing": light_tracing_workload(cpu=not args.no_cpu_baseline)},
                   lambda: {"denoise": denoise_workload()}):
            try:
                workloads.update(fn())
            except Exception as ex:  # reported, never fatal for the GPU line
                workloads.setdefault("errors", []).append(str(ex))

    rmse = None
    if rank == 0 and world == 1 and not args.no_rmse:
        try:
            rmse = time_to_rmse()
        except Exception as ex:  # reported, never fatal for the GPU line
            rmse = {"error": str(ex)}

    if rank == 0:
        base = None
        if world == 1 and not args.no_cpu_baseline:
            try:
                base = cpu_baseline()
            except Exception as ex:  # reported, never fatal for the GPU line
                base = {"error": str(ex)}
        launches_per_step = launches / args.steps
        # the metric's own targets, each on the workload it is stated for
        targets = {}
        tpw = workloads.get("terrain_pt") if isinstance(workloads, dict) else None
        if tpw:
            targets["terrain_pt_segments_per_s"] = {
                "value": tpw["segments_per_s"], "target": 2.0, "unit": UNIT, "higher_is_better": True,
                "workload": f"{tpw['workload']}, {tpw['triangles']} triangles"}
        if isinstance(rmse, dict) and "guided_over_plain" in rmse:
            targets["guided_over_plain_time_to_1pct"] = {
                "value": rmse["guided_over_plain"], "target": 0.5, "unit": "ratio of device seconds",
                "higher_is_better": False, "workload": rmse["scene"],
                "per_pixel_ratio": rmse.get("guided_over_plain_pixel")}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"Cornell box PT {W}x{H}, {SPP_PER_STEP} spp per step, max path length "
                                   f"{MAX_PATH_LENGTH}, 4 hero wavelengths, MIS NEE, FP64 film",
                       "scene_triangles": ctx.stats()["numTriangles"],
                       "l2": f"working set > L2: {launch_opts['maxPathsInFlight']} path slots x ~200 B of SoA "
                             f"path state per launch",
                       "launch": {"paths_in_flight": launch_opts["maxPathsInFlight"],
                                  "blocks_per_sm": launch_opts["blocksPerSM"],
                                  "chosen_by": chosen},
                       "parallelism": f"replica render per GPU + NCCL film all-reduce" if world > 1 else "1 GPU"},
            "segments_per_step": seg_total / args.steps,
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(param_bytes / args.steps),
                    "d2h_bytes_per_step": W * H * 16},
            "roofline": roofline,
            "cpu_baseline": base,
            "gpu_launches": int(launches),
            "gpu_launches_per_step": launches_per_step,
            "clocks": clocks.summary(),
            "targets": targets,
            "time_to_rmse": rmse,
            "workloads": workloads,
        }
        print(json.dumps(line))
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
