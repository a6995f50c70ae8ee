"""Benchmark of the volumetric path-tracing hot path on B200.

Workload (the dense multi-tracker configuration): 512^3 fp32 fBm Perlin cloud (seed 2, 6 octaves,
lacunarity 2, gain 0.5, ~35% empty), unit cube, extinction 1000, albedo 0.99, HG g = 0.85, sun 5
plus constant sky 0.2, pinhole camera 60 deg at distance 2, 1024x1024, max 128 bounces.  One step =
one render_frame of SPP_PER_STEP 1-spp frames (1024^2 * SPP_PER_STEP camera paths) with delta
tracking; the other trackers are timed on the same steps (per_tracker) and their images are compared
with an FP64-accumulated 16384-spp delta-tracking render.  The grid (512 MiB) is
larger than L2, so no flush is needed between steps.

`python bench.py --gpus N --steps K --warmup W` prints one JSON line (rank 0).  Under torchrun each
rank renders its own frame range of the image (weak scaling, no collective on the data path).
`--impl reference` times the CPU oracle on this host (bounded sample of the same workload).
"""
from __future__ import annotations

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
sys.path.insert(0, ROOT)

METRIC = "path samples/s per tracker"
UNIT = "path samples/s"
GRID = 512
RES = 1024
SPP_PER_STEP = 64
MAX_BOUNCES = 128
EXTINCTION = 1000.0
SEED = 2
TRACKERS = {"delta": 0, "ratio": 2, "decomposition": 3, "residual_ratio": 4, "nee": 5, "residual_ratio_unbiased": 9}
BYTES_PER_LOOKUP = 32  # one 32-byte sector per uncoalesced density gather
# delta tracking reads the density through the grid's 3D texture object (1) or by global loads (0);
# both read the same texels; the bench's fetch_paths_delta leg times the two
DENSITY_TEXTURE = 1
# per-lane refill schedule: a warp takes new paths once this many of its lanes wait (the library's
# default; refill_min_lanes_delta times 1, 2, 4 and 8)
REFILL_MIN_LANES = 4
# DRAM read + write bytes of one headline launch (64 spp of the 1024^2 image on the 512^3 cloud, density
# through the texture object), from one ncu capture of that launch
# (profiles/trace_refill_delta_512_1024_64spp.md): 37.09 GB, 553 B per path
NCU_DRAM_BYTES_PER_PATH = (35.250e9 + 1.844e9) / (1024 * 1024 * 64)


def tensor_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["bf16_tflops"]), "measured cuBLAS bf16 burst"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def gather_rates(lib, stream):
    """Random 32-byte-sector gather rates (GB/s of sectors) of this GPU: a 512 MiB buffer (HBM) and a
    32 MiB buffer (L2), timed with CUDA events after a warm-up launch."""
    import ctypes
    import torch
    out = {}
    sink = torch.zeros(1, device="cuda")
    cs = ctypes.c_void_p(stream.cuda_stream)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    for name, mib in (("hbm", 512), ("l2", 32)):
        buf = torch.rand(mib * 1024 * 1024 // 4, device="cuda")
        blocks, loads = sms * 8, 512
        for _ in range(2):
            vpt_check(lib.vpt_gather_bench(ctypes.c_void_p(buf.data_ptr()), buf.numel() * 4, blocks, loads, 7,
                                           ctypes.c_void_p(sink.data_ptr()), cs))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for r in range(5):
            vpt_check(lib.vpt_gather_bench(ctypes.c_void_p(buf.data_ptr()), buf.numel() * 4, blocks, loads, 11 + r,
                                           ctypes.c_void_p(sink.data_ptr()), cs))
        e1.record(stream)
        torch.cuda.synchronize()
        sectors = 5.0 * blocks * 256 * loads
        out[name] = sectors * BYTES_PER_LOOKUP / (e0.elapsed_time(e1) / 1e3) / 1e9
        del buf
    return out


def run_streaming(lib, stream):
    """The builders and image filters around the tracer, each on inputs larger than L2, timed with
    CUDA events (one warm-up call, then the mean of 3): algorithmic bytes (every input read once,
    every output written once) / time against the measured HBM copy peak."""
    import ctypes
    import torch
    cs = ctypes.c_void_p(stream.cuda_stream)
    peak, peak_kind = peaks()
    out = {"peak_gbs": peak, "peak_kind": peak_kind}

    def p(t):
        return ctypes.c_void_p(t.data_ptr())

    def timed(name, fn, nbytes, work):
        fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(3):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 3
        out[name] = {"work": work, "bytes": int(nbytes), "ms": ms, "gbs": nbytes / (ms / 1e3) / 1e9,
                     "frac_of_hbm_peak": nbytes / (ms / 1e3) / 1e9 / peak}

    n = 512
    dens = torch.rand(n * n * n, device="cuda")
    sv = 8
    g = n // sv
    smin, smax, savg = (torch.empty(g ** 3, device="cuda") for _ in range(3))
    socc = torch.empty(g ** 3, dtype=torch.uint8, device="cuda")
    timed("supervoxel_grid", lambda: vpt_check(lib.vpt_build_supervoxel_grid(
        p(dens), n, n, n, sv, 1, p(smin), p(smax), p(savg), p(socc), cs)),
        dens.numel() * 4 + g ** 3 * 13, f"{n}^3 grid, 8^3 supervoxels with halo: min/max/mean/occupancy")
    occ = torch.empty(g ** 3, dtype=torch.uint8, device="cuda")
    dens.zero_()  # an empty grid: every block reads all its voxels (an occupied block stops at its first hit)
    timed("occupancy_grid", lambda: vpt_check(lib.vpt_build_occupancy_grid(
        p(dens), n, n, n, 8, 1, ctypes.c_float(0.0), p(occ), cs)),
        dens.numel() * 4 + g ** 3, f"{n}^3 empty grid (the worst case), 8^3 blocks with a one-voxel halo")
    del dens, smin, smax, savg, socc, occ

    W = H = 2048
    color, pos, nrm = (torch.rand(H * W * 4, device="cuda") for _ in range(3))
    dst = torch.empty_like(color)
    iters = 5
    timed("eaw", lambda: vpt_check(lib.vpt_eaw_denoise_rgba(
        p(color), p(pos), p(nrm), W, H, iters, ctypes.c_float(0.5), ctypes.c_float(0.5), ctypes.c_float(0.5), 1,
        p(dst), cs)),
        iters * W * H * (3 * 16 + 16), f"{W}x{H} RGBA, {iters} a-trous iterations (colour, position, normal in, "
                                      "colour out per iteration)")
    del pos, nrm, dst
    k = 5
    logits = torch.rand(1 * k * k * H * W, device="cuda")
    img = color[:3 * H * W].contiguous()
    kout = torch.empty(3 * H * W, device="cuda")
    timed("kpn_apply", lambda: vpt_check(lib.vpt_kpn_apply(
        p(img), p(logits), 1, 3, H, W, H, W, k, 1, p(kout), cs)),
        (k * k + 3 + 3) * 4 * H * W, f"{W}x{H}, 3 channels, {k}x{k} per-pixel kernels with the tap softmax fused")
    return out


def vpt_check(st):
    if st != 0:
        raise RuntimeError(f"vpt_gather_bench failed with status {st}")


def workload_config(n_gpus):
    return {"workload": f"dense {GRID}^3 fBm cloud, {RES}x{RES}, {SPP_PER_STEP} spp/step, delta tracking "
                        f"(+ratio/decomposition/residual-ratio/NEE timed separately)",
            "grid": GRID, "image": RES, "spp_per_step": SPP_PER_STEP, "max_bounces": MAX_BOUNCES,
            "extinction": EXTINCTION, "albedo": 0.99, "g": 0.85, "interpolation": "stochastic",
            "l2": "grid 512 MiB > L2 126 MB: inputs larger than L2, no flush",
            "parallelism": f"spp-sharded x{n_gpus}" if n_gpus > 1 else "single GPU"}


def sun_dir(seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=3)
    v[1] = abs(v[1]) + 0.5
    return (v / np.linalg.norm(v)).tolist()


def camera_pos(seed):
    rng = np.random.default_rng(seed + 1000)
    a = rng.uniform(0, 2 * math.pi)
    return [2.0 * math.sin(a), 0.4, 2.0 * math.cos(a)]


class Clocks:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def setup_scene(vpt, rank):
    vpt.set_max_grid_extent(0.5)
    vpt.generate_fbm_cloud(GRID, seed=SEED)
    vpt.set_extinction_scale(EXTINCTION)
    vpt.set_scattering_albedo([0.99, 0.99, 0.99])
    vpt.set_phase_g(0.85)
    vpt.set_use_builtin_environment_map("Constant Sky + Sun")
    vpt.set_sky_color([0.2, 0.2, 0.2])
    vpt.set_sun(sun_dir(SEED), [5.0, 5.0, 5.0])
    vpt.set_camera_position(camera_pos(SEED))
    vpt.set_camera_target([0.0, 0.0, 0.0])
    vpt.set_camera_fovy(60.0)
    vpt.set_max_bounces(MAX_BOUNCES)
    vpt.set_grid_interpolation("Stochastic")
    vpt.set_denoiser("None")
    # distinct paths per rank: the seed of a path is (frame * W * H + pixel + offset) mod 2^32
    # (Clouds.glsl:80-84), so frame indices repeat every 2^32 / (W * H) frames (4096 at 1024^2); a
    # per-rank seed offset that is not a multiple of W * H gives every rank its own seeds per pixel
    vpt.set_seed_offset(rank_seed_offset(rank))


def rank_seed_offset(rank):
    """Seed offset of a rank: a multiple of W*H/8, distinct modulo W*H for up to 8 ranks."""
    return (rank % 8) * (RES * RES // 8)


def run_ours(args):
    import torch
    from cloudrendering_b200 import vpt, _lib

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    lib = _lib.load()
    vpt.initialize()
    ctx = vpt.context_handle()
    setup_scene(vpt, rank)
    _lib.check(lib.vpt_set_option(ctx, b"density_texture", float(DENSITY_TEXTURE)), "density_texture", ctx)
    _lib.check(lib.vpt_set_option(ctx, b"refill_min_lanes", float(REFILL_MIN_LANES)), "refill_min_lanes", ctx)
    stream = torch.cuda.current_stream()
    ctypes_stream = __import__("ctypes").c_void_p(stream.cuda_stream)
    img = torch.zeros((4, RES, RES), dtype=torch.float32, device="cuda")

    def render_step():
        _lib.check(lib.vpt_render_frames(ctx, SPP_PER_STEP, ctypes_stream), "render", ctx)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        if world == 1:
            return v
        import torch.distributed as dist
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    vpt.set_vpt_mode_from_name("Delta Tracking")
    vpt.render_frame(img, 1)
    for _ in range(args.warmup):
        render_step()
    barrier()
    vpt.reset_stats()
    launches0 = lib.vpt_kernel_launch_count()
    clocks = Clocks(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    ev0.record(stream)
    for _ in range(args.steps):
        render_step()
    ev1.record(stream)
    barrier()
    clock_info = clocks.stop()
    ms_total = max_over_ranks(ev0.elapsed_time(ev1))
    launches = lib.vpt_kernel_launch_count() - launches0
    st = vpt.get_stats()
    _lib.check(lib.vpt_synchronize(ctx, ctypes_stream), "sync", ctx)
    paths_per_rank = RES * RES * SPP_PER_STEP * args.steps
    total_paths = paths_per_rank * world
    value = total_paths / (ms_total / 1e3)
    lookups = st["density_lookups"]
    ms_per_launch = ms_total / args.steps
    achieved = (lookups / args.steps) * BYTES_PER_LOOKUP / (ms_per_launch / 1e3) / 1e9
    peak, peak_kind = peaks()

    # per tracker: rates on 64-spp steps and the error of each tracker's image against an
    # FP64-accumulated 16384-spp delta-tracking render of the same scene
    per_tracker, reference_render = run_trackers(vpt, lib, ctx, img, stream, ctypes_stream, barrier, max_over_ranks,
                                                 rank, world, args.workload == "small")

    # schedule comparison for delta tracking (the reason the refill schedule is the default)
    schedules = {}
    vpt.set_vpt_mode_from_name("Delta Tracking")
    for sched, label in ((0, "tiles"), (1, "persistent_warp_batches"), (2, "per_lane_refill")):
        _lib.check(lib.vpt_set_option(ctx, b"schedule", float(sched)), "schedule", ctx)
        vpt.render_frame(img, 1)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _lib.check(lib.vpt_render_frames(ctx, SPP_PER_STEP, ctypes_stream), "render", ctx)
        e1.record(stream)
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1))
        schedules[label] = RES * RES * SPP_PER_STEP * world / (ms / 1e3)
    _lib.check(lib.vpt_set_option(ctx, b"schedule", 2.0), "schedule", ctx)

    # density fetch path for delta tracking: plain global loads of the x-fastest grid against the 3D
    # texture object (block layout, bounds test in the texture unit); both read the same texels
    fetch = {}
    for tex, label in ((0, "global_loads"), (1, "texture_object"), (DENSITY_TEXTURE, "selected")):
        _lib.check(lib.vpt_set_option(ctx, b"density_texture", float(tex)), "density_texture", ctx)
        vpt.render_frame(img, 1)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(3):
            _lib.check(lib.vpt_render_frames(ctx, SPP_PER_STEP, ctypes_stream), "render", ctx)
        e1.record(stream)
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1)) / 3
        fetch[label] = RES * RES * SPP_PER_STEP * world / (ms / 1e3)
    fetch["selected"] = "texture_object" if DENSITY_TEXTURE else "global_loads"
    _lib.check(lib.vpt_set_option(ctx, b"density_texture", float(DENSITY_TEXTURE)), "density_texture", ctx)

    # refills taken once k lanes of a warp wait (the film is written when each path ends; the paths are
    # the same for every k)
    refill = {}
    for k in (1, 2, 4, 8):
        _lib.check(lib.vpt_set_option(ctx, b"refill_min_lanes", float(k)), "refill_min_lanes", ctx)
        vpt.render_frame(img, 1)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(3):
            _lib.check(lib.vpt_render_frames(ctx, SPP_PER_STEP, ctypes_stream), "render", ctx)
        e1.record(stream)
        barrier()
        refill[str(k)] = RES * RES * SPP_PER_STEP * world / (max_over_ranks(e0.elapsed_time(e1)) / 3 / 1e3)
    _lib.check(lib.vpt_set_option(ctx, b"refill_min_lanes", float(REFILL_MIN_LANES)), "refill_min_lanes", ctx)
    refill["selected"] = REFILL_MIN_LANES


    # end to end through the public API: host grid -> device, render, result -> host
    vpt.set_vpt_mode_from_name("Delta Tracking")
    grid_host = torch.empty((GRID, GRID, GRID), dtype=torch.float32).pin_memory()
    _lib.check(lib.vpt_get_dense_grid(ctx, __import__("ctypes").c_void_p(grid_host.data_ptr()), 0), "get grid", ctx)
    out_cpu = torch.zeros((4, RES, RES), dtype=torch.float32)
    e2e_steps = max(1, min(args.steps, 3))
    vpt.set_density_field(grid_host)  # untimed warm-up step of this path (host-side buffers, first copies)
    vpt.render_frame(out_cpu, SPP_PER_STEP)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        vpt.set_density_field(grid_host)
        res = vpt.render_frame(out_cpu, SPP_PER_STEP)
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e = {"value": RES * RES * SPP_PER_STEP * e2e_steps * world / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": GRID ** 3 * 4, "d2h_bytes_per_step": int(res.numel() * 4),
           "path": "vpt.set_density_field(pinned host grid) + vpt.render_frame(cpu tensor)"}

    gather = gather_rates(lib, stream)
    streaming = run_streaming(lib, stream) if rank == 0 else None
    gather_roofline = {"unit": "GB/s", "achieved": achieved, "hbm_random_sector": gather["hbm"],
                       "l2_random_sector": gather["l2"], "frac_of_hbm_random_sector": achieved / gather["hbm"],
                       "frac_of_l2_random_sector": achieved / gather["l2"],
                       "note": "same achieved bytes as roofline, against this GPU's random 32 B sector gather rate "
                               "(vpt_gather_bench, measured in this run)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(lib, ctx, vpt)

    sparse = None
    if not args.no_sparse:
        sparse = run_sparse(vpt, lib, ctx, stream, ctypes_stream, barrier, max_over_ranks, world)
    batch = None
    if not args.no_batch:
        batch = run_batch(lib, stream, ctypes_stream, barrier, max_over_ranks, world)
    learned = None
    if not args.no_learned:
        learned = run_learned(vpt, lib, ctx, args.workload == "small")

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded fBm Perlin cloud)",
            "config": workload_config(world),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": NCU_DRAM_BYTES_PER_PATH * RES * RES * SPP_PER_STEP if args.workload == "full" else None,
                         "limiter": "instruction issue at low SIMT efficiency (70 % issue active, 13.6 of 32 lanes per "
                                    "instruction, DRAM 10 % busy; profiles/trace_refill_delta_512_1024_64spp.md)",
                         "note": f"algorithmic bytes = density lookups x {BYTES_PER_LOOKUP} B sector; peak {peak_kind} "
                                 "HBM copy; traffic = ncu dram read + write bytes of this launch"},
            "lookups_per_s": lookups / (ms_total / 1e3) * world,
            "lookups_per_path": lookups / max(1, st["paths"]),
            "gather_roofline": gather_roofline,
            "per_tracker": per_tracker, "tracker_reference_render": reference_render, "schedules_delta": schedules, "fetch_paths_delta": fetch, "refill_min_lanes_delta": refill, "streaming_kernels": streaming, "e2e": e2e, "gpu_launches": int(launches), "clocks": clock_info,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        if sparse is not None:
            line["sparse_nanovdb"] = sparse
        if batch is not None:
            line["batched_scenes"] = batch
        if learned is not None:
            line["learned_denoiser"] = learned
        print(json.dumps(line), flush=True)
    vpt.cleanup()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


TRACKER_STEPS = 4  # 4 steps of SPP_PER_STEP frames: 256 spp per tracker
TRACKER_STEP_BUDGET_MS = 4000.0
REF_SPP = 16384
RELMSE_EPS = 1e-2


def independent_passes(width, height, spp):
    """(seed offset, frames) passes whose paths are independent of a render at seed offset 0.

    The seed of a path is (frame * W * H + pixel + offset) mod 2^32 (Clouds.glsl:80-84), so one seed
    offset yields at most 2^32 / (W * H) distinct frames per pixel (4096 at 1024^2).  Offsets that are
    multiples of W * H / 8 other than 0 mod W * H give each pixel seeds that neither repeat across the
    passes nor coincide with the seeds of that pixel at offset 0."""
    period = (1 << 32) // (width * height)
    passes, k = [], 1
    while spp > 0:
        n = min(spp, period)
        passes.append((k * (width * height // 8), n))
        spp -= n
        k += 1
    if len(passes) > 7:
        raise ValueError("too many samples for independent passes at this image size")
    return passes


def film_moments_f64(lib, ctx, n, stream):
    """(sum, sum of squares) of the accumulated frames' radiance, float64 [H*W*3] on the GPU."""
    import ctypes
    import torch
    from cloudrendering_b200 import _lib
    s = torch.empty(n * 3, dtype=torch.float64, device="cuda")
    q = torch.empty_like(s)
    _lib.check(lib.vpt_read_statistics(ctx, ctypes.c_void_p(s.data_ptr()), ctypes.c_void_p(q.data_ptr()), 1,
                                       ctypes.c_void_p(stream.cuda_stream)), "statistics", ctx)
    return s, q


def run_trackers(vpt, lib, ctx, img, stream, ctypes_stream, barrier, max_over_ranks, rank, world, small):
    """Each tracker on the bench scene: TRACKER_STEPS timed steps of SPP_PER_STEP frames (path samples/s,
    density lookups/s), then its image (TRACKER_STEPS * SPP_PER_STEP spp) against the FP64 16384-spp
    delta-tracking render: relMSE = mean((x - ref)^2 / (ref^2 + RELMSE_EPS)) over pixels and channels,
    and per-pixel z-scores (x - ref) / sqrt(var_x / n_x + var_ref / n_ref) from each render's own
    per-pixel sample variance, with the image mean's deviation in standard errors."""
    import torch
    from cloudrendering_b200 import _lib
    ref_spp = 1024 if small else REF_SPP
    n_pix = RES * RES
    vpt.set_vpt_mode_from_name("Delta Tracking")
    vpt.set_use_isosurfaces(False)
    vpt.set_collect_statistics(True)
    t0 = time.perf_counter()
    rs = rq = None
    for offset, frames in independent_passes(RES, RES, ref_spp):
        vpt.set_seed_offset(offset)
        vpt.set_frame_index(0)
        left = frames
        while left > 0:
            k = min(256, left)
            _lib.check(lib.vpt_render_frames(ctx, k, ctypes_stream), "render", ctx)
            left -= k
        s_, q_ = film_moments_f64(lib, ctx, n_pix, stream)
        rs, rq = (s_, q_) if rs is None else (rs + s_, rq + q_)
    torch.cuda.synchronize()
    vpt.set_seed_offset(rank_seed_offset(rank))
    ref_s = time.perf_counter() - t0
    ref_mean = rs / ref_spp
    ref_var = torch.clamp(rq / ref_spp - ref_mean * ref_mean, min=0.0) * (ref_spp / (ref_spp - 1))
    out = {}
    # delta and next event tracking with isosurfaces at density 0.5 (Lambertian surfaces, trilinear
    # lookups; next event tracking with surface light samples) make a different image: their rates only
    for name, mode in list(TRACKERS.items()) + [("nee_empty_space_skipping", 5), ("delta_isosurfaces", 0),
                                                ("nee_isosurfaces", 5)]:
        iso = name in ("delta_isosurfaces", "nee_isosurfaces")
        vpt.set_vpt_mode(mode)
        vpt.set_use_isosurfaces(iso)
        # next event tracking whose shadow rays skip the occupancy grid's empty 8^3 blocks
        vpt.set_use_empty_space_skipping(name == "nee_empty_space_skipping")
        vpt.set_iso_value(0.5)
        vpt.set_frame_index(0)
        _lib.check(lib.vpt_render_frames(ctx, 1, ctypes_stream), "warm-up", ctx)
        vpt.set_frame_index(0)
        barrier()
        vpt.reset_stats()
        # up to TRACKER_STEPS steps; a tracker slower than TRACKER_STEP_BUDGET_MS per step stops after the
        # steps that fit (at least one), and its error is stated at the samples it rendered
        steps, ms = 0, 0.0
        while steps < (1 if iso else TRACKER_STEPS):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            _lib.check(lib.vpt_render_frames(ctx, SPP_PER_STEP, ctypes_stream), "render", ctx)
            e1.record(stream)
            barrier()
            ms += max_over_ranks(e0.elapsed_time(e1))
            steps += 1
            if ms > TRACKER_STEP_BUDGET_MS:
                break
        st = vpt.get_stats()
        row = {"path_samples_per_s": n_pix * SPP_PER_STEP * steps * world / (ms / 1e3),
               "lookups_per_path": st["density_lookups"] / max(1, st["paths"]),
               "lookups_per_s": st["density_lookups"] * world / (ms / 1e3),
               "ms_per_step": ms / steps, "spp_per_step": SPP_PER_STEP}
        if not iso:
            spp = steps * SPP_PER_STEP
            s, q = film_moments_f64(lib, ctx, n_pix, stream)
            m = s / spp
            var = torch.clamp(q / spp - m * m, min=0.0) * (spp / (spp - 1))
            finite = torch.isfinite(m).view(-1, 3).all(dim=1).repeat_interleave(3)
            nonfinite = int((~finite).sum()) // 3
            mf, rf, vf, rvf = m[finite], ref_mean[finite], var[finite], ref_var[finite]
            rel = float(((mf - rf) ** 2 / (rf ** 2 + RELMSE_EPS)).mean())
            se = torch.sqrt(vf / spp + rvf / ref_spp)
            z = torch.where(se > 0, (mf - rf) / torch.where(se > 0, se, torch.ones_like(se)), torch.zeros_like(se))
            za = z.abs()
            mc = mf.view(-1, 3).mean(dim=0)
            rc = rf.view(-1, 3).mean(dim=0)
            npx = mf.numel() // 3
            se_mean = torch.sqrt(vf.view(-1, 3).mean(dim=0) / (spp * npx) + rvf.view(-1, 3).mean(dim=0) / (ref_spp * npx))
            row.update({"spp": spp, "relmse_vs_fp64_16k": rel, "relmse_eps": RELMSE_EPS,
                        # error times render time: constant for an unbiased estimator (relMSE ~ 1/spp), so
                        # trackers compare at equal time
                        "relmse_x_ms": rel * ms,
                        "nonfinite_pixels": nonfinite,
                        "z_vs_fp64_16k": {"max_abs": float(za.max()), "frac_abs_gt_3": float((za > 3).float().mean()),
                                          "frac_abs_gt_4": float((za > 4).float().mean()),
                                          "normal_frac_abs_gt_3": 0.0027, "normal_frac_abs_gt_4": 6.3e-5},
                        "image_mean_dev_in_se": float(((mc - rc).abs() / se_mean).max()),
                        "image_mean": [float(v) for v in mc]})
        out[name] = row
    vpt.set_use_isosurfaces(False)
    vpt.set_use_empty_space_skipping(False)
    vpt.set_collect_statistics(False)
    vpt.set_frame_index(0)
    reference = {"tracker": "delta", "spp": ref_spp, "accumulation": "fp64", "seconds": ref_s,
                 "passes": [{"seed_offset": o, "frames": f} for o, f in independent_passes(RES, RES, ref_spp)],
                 "image_mean": [float(v) for v in ref_mean.view(-1, 3).mean(dim=0)],
                 "z_note": "per pixel-channel (x - ref) / sqrt(var_x / n_x + var_ref / n_ref) with sample variances; "
                           "heavy-tailed pixels (the sun lobe) make the largest |z| unreliable at 256 spp, so the "
                           "tail fractions are reported beside the normal distribution's"}
    return out, reference


# Learned denoiser: a kernel-predicting U-Net (widths 32-64-96-128-160, 13x13 kernels) trained on the
# GPU by this package's tcgen05 kernels on tracer-generated pairs (512 seeded cloud scenes at 256^2:
# noisy renders at 1..256 spp with albedo / normal / depth / transmittance features against 2048-spp
# targets from disjoint frames; Adam, batch 8, 6000 steps, learning rate cosine-annealed from 5e-4 to
# 1e-5), then the time each method needs to reach relMSE <= 1e-3 on held-out scenes (256^3 clouds,
# 512^2, max 128 bounces) against their FP64-accumulated 16384-spp renders: plain accumulation, EAW
# (iteration count 1..5 chosen per sample count by the lowest error, i.e. tuned with the reference in
# hand), SVGF (one 1-spp frame per call, history carried between calls) and the learned denoiser.
LEARNED = dict(scenes=512, size=256, spp_levels=(1, 2, 4, 8, 16, 64, 256), target_spp=2048, steps=6000, batch=8,
               lr=5e-4, lr_end=1e-5, kernel_size=13, grid=128)
EVAL = dict(seeds=(77777, 77778, 77779, 77780), res=512, grid=256, max_bounces=128, ref_spp=16384,
            levels=(1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096), target=1e-3)


def time_to_target(spp, err, time_of, target, extrapolate):
    """Samples and time at which err(spp) first reaches target (log-log interpolation between the
    bracketing levels); for unbiased accumulation beyond the last level, err ~ 1/spp."""
    for i, (n, r) in enumerate(zip(spp, err)):
        if r <= target:
            if i == 0:
                ns = float(n)
            else:
                n0, r0 = spp[i - 1], err[i - 1]
                t = (math.log(target) - math.log(r0)) / (math.log(r) - math.log(r0))
                ns = math.exp(math.log(n0) + t * (math.log(n) - math.log(n0)))
            return {"spp": ns, "ms": time_of(ns), "extrapolated": False}
    if not extrapolate:
        return {"spp": None, "ms": None, "extrapolated": False}
    ns = spp[-1] * err[-1] / target
    return {"spp": ns, "ms": time_of(ns), "extrapolated": True}


def run_learned(vpt, lib, ctx, small):
    import ctypes
    import torch
    from cloudrendering_b200 import learned_denoiser as ld

    cfg, ev = dict(LEARNED), dict(EVAL)
    if small:
        cfg.update(scenes=8, size=128, steps=300, target_spp=512, lr_end=None)
        ev.update(seeds=(77777,), res=256, grid=128, ref_spp=4096, levels=(1, 2, 4, 8, 16, 32, 64, 128, 256, 512))
    stream = torch.cuda.current_stream()
    cs = ctypes.c_void_p(stream.cuda_stream)
    data = ld.TrainingSet(vpt, cfg["scenes"], cfg["size"], cfg["spp_levels"], cfg["target_spp"], grid=cfg["grid"])
    net = ld.KpnUNet(seed=0, kernel_size=cfg["kernel_size"])
    # training-step throughput (convolutions forward + input gradient + weight gradient)
    rng = np.random.default_rng(0)
    b = data.batch(rng, cfg["batch"])
    for _ in range(3):
        net.train_step(b, 0.0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k0 = lib.vpt_kernel_launch_count()
    e0.record(stream)
    for _ in range(10):
        net.train_step(b, 0.0)
    e1.record(stream)
    torch.cuda.synchronize()
    step_ms = e0.elapsed_time(e1) / 10
    launches_per_step = (lib.vpt_kernel_launch_count() - k0) / 10
    P0 = cfg["batch"] * cfg["size"] ** 2
    conv_flop = sum(2 * 9 * L["cin"] * L["cout"] * (P0 >> (2 * L["level"])) * (2 if L["name"] == "enc0a" else 3)
                    for L in net.layers)
    net = ld.KpnUNet(seed=0, kernel_size=cfg["kernel_size"])
    hist = ld.train(net, data, cfg["steps"], cfg["batch"], cfg["lr"], seed=1, lr_end=cfg.get("lr_end"))

    def eval_scene(seed):
        """One held-out scene: its FP64 reference, every method's error curve and time to target."""
        # held-out scene: FP64 reference, then the error curves
        sc = ld.sample_scene(seed)
        ld.setup_scene(vpt, sc, grid=ev["grid"], max_bounces=ev["max_bounces"])
        R = ev["res"]
        img = torch.zeros((3, R, R), dtype=torch.float32, device="cuda")

        def frame_ms(frames):
            vpt.render_frame(img, 2)
            a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            _lib_check(lib.vpt_render_frames(ctx, frames, cs))
            c.record(stream)
            torch.cuda.synchronize()
            return a.elapsed_time(c) / frames

        def _lib_check(st):
            vpt._lib.check(st, "render", ctx)

        t_ref = time.perf_counter()
        ref = None
        for offset, frames in independent_passes(R, R, ev["ref_spp"]):
            vpt.set_seed_offset(offset)
            vpt.set_frame_index(0)
            left = frames
            while left > 0:
                k = min(256, left)
                vpt.render_frame(img, k)
                left -= k
            part = vpt.get_film_sum(R, R).cuda()
            ref = part if ref is None else ref + part
        ref = ref / float(ev["ref_spp"])
        ref_s = time.perf_counter() - t_ref
        vpt.set_seed_offset(0)
        vpt.set_frame_index(0)
        ms_plain = frame_ms(64)
        vpt.set_use_feature_maps(["Albedo", "Normal", "Depth", "Transmittance"])
        vpt.set_denoiser("Edge-Avoiding À-Trous Wavelet Transform")
        vpt.set_denoiser_property("iterations", "1")
        ms_feat = frame_ms(64)  # a frame with the feature pass
        # each denoiser with its own best feature setting: EAW's edge-stopping weights want feature maps
        # accumulated over every frame (as the reference renders them); the learned denoiser reads feature
        # maps accumulated over the first FEATURE_FRAMES frames (as it was trained), and later frames are
        # traced without the feature pass
        kf = ld.FEATURE_FRAMES

        def render_ms(spp):
            return min(spp, kf) * ms_feat + max(0.0, spp - kf) * ms_plain

        def timed(fn):
            a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            r = fn()
            c.record(stream)
            torch.cuda.synchronize()
            return r, a.elapsed_time(c)

        rows = [{"spp": n} for n in ev["levels"]]
        eaw_ms, net_ms = {}, []
        # pass 1: plain accumulation and EAW (features every frame)
        vpt.set_frame_index(0)
        done = 0
        for row in rows:
            n = row["spp"]
            vpt.render_frame(img, n - done)
            done = n
            plain = (vpt.get_film_sum(R, R).cuda() / n).float().contiguous()
            row["plain"] = ld.relmse(plain, ref)
            best = None
            for it in (1, 2, 3, 4, 5):
                vpt.set_denoiser_property("iterations", str(it))
                d, ms = timed(lambda: vpt.get_feature_map(img, 0))
                eaw_ms.setdefault(it, []).append(ms)
                r = ld.relmse(d, ref)
                if best is None or r < best[0]:
                    best = (r, it)
            row["eaw"], row["eaw_iterations"] = best
        # pass 2: the learned denoiser (the same frames: identical film, features over the first kf frames),
        # replayed from a CUDA graph captured for this image size
        dgraph = net.graph(1, R, R)
        vpt.set_denoiser("None")
        vpt.set_feature_frame_limit(kf)
        vpt.set_frame_index(0)
        done = 0
        for row in rows:
            n = row["spp"]
            vpt.render_frame(img, n - done)
            done = n
            plain = (vpt.get_film_sum(R, R).cuda() / n).float().contiguous()

            noise = torch.full((1,), 1.0 / math.sqrt(n), device="cuda")

            def learned_once():  # the renderer's feature planes go straight into the graph's inputs
                return dgraph.from_renderer(vpt, plain, noise)[0]
            den, ms = timed(learned_once)
            net_ms.append(ms)
            row["learned"] = ld.relmse(den, ref)
        vpt.set_feature_frame_limit(0)
        # pass 3: SVGF as the reference runs it: every call traces one 1-spp frame with its feature maps,
        # and the filter carries its colour / moments history from call to call (static camera); the error
        # after n calls is SVGF's estimate from n samples
        vpt.set_denoiser("SVGF")
        vpt.set_frame_index(0)
        svgf_ms = []
        done = 0
        for row in rows:
            n = row["spp"]
            out = None
            while done < n:
                out, ms = timed(lambda: vpt.render_frame(img, 1))
                svgf_ms.append(ms)
                done += 1
            row["svgf"] = ld.relmse(out[:3].float().contiguous(), ref)
        vpt.set_denoiser("None")
        vpt.set_use_feature_maps([])
        net.check_errors()
        spp = [r["spp"] for r in rows]
        svgf_cost = statistics.median(svgf_ms)  # one traced frame with features + the filter
        svgf_t = time_to_target(spp, [r["svgf"] for r in rows], lambda s: s * svgf_cost, ev["target"], False)
        eaw_cost = statistics.median(sum(v) / len(v) for v in eaw_ms.values())
        net_cost = statistics.median(net_ms)
        plain_t = time_to_target(spp, [r["plain"] for r in rows], lambda s: s * ms_plain, ev["target"], True)
        eaw_t = time_to_target(spp, [r["eaw"] for r in rows], lambda s: s * ms_feat + eaw_cost, ev["target"], False)
        learned_t = time_to_target(spp, [r["learned"] for r in rows], lambda s: render_ms(s) + net_cost, ev["target"],
                                   False)
        return {"seed": seed, "rows": rows, "plain": plain_t, "eaw_tuned": eaw_t, "svgf": svgf_t,
                "learned": learned_t, "ms_plain": ms_plain, "ms_feat": ms_feat, "eaw_cost": eaw_cost,
                "net_cost": net_cost, "svgf_cost": svgf_cost, "ref_s": ref_s, "kf": kf, "R": R}

    scenes = [eval_scene(sd) for sd in ev["seeds"]]
    speedups = [e["eaw_tuned"]["ms"] / e["learned"]["ms"] for e in scenes
                if e["learned"]["ms"] and e["eaw_tuned"]["ms"]]
    first = scenes[0]
    rows, plain_t, eaw_t, svgf_t, learned_t = (first["rows"], first["plain"], first["eaw_tuned"], first["svgf"],
                                               first["learned"])
    ms_plain, ms_feat, kf, R = first["ms_plain"], first["ms_feat"], first["kf"], first["R"]
    eaw_cost, net_cost, svgf_cost, ref_s = first["eaw_cost"], first["net_cost"], first["svgf_cost"], first["ref_s"]
    peak, peak_kind = tensor_peak()
    out = {
        "workload": (f"KPN U-Net {'-'.join(map(str, net.widths))}, {cfg['kernel_size']}x{cfg['kernel_size']} kernels, "
                     f"trained {cfg['steps']} steps (batch {cfg['batch']} x {cfg['size']}^2, {cfg['scenes']} scenes, "
                     f"inputs {cfg['spp_levels']} spp vs {cfg['target_spp']}-spp targets); held-out scene seed "
                     f"{ev['seeds'][0]} (curves; {len(ev['seeds'])} seeds for the median speed-up) {ev['grid']}^3 at {R}^2 vs its "
                     f"FP64 {ev['ref_spp']}-spp render"),
        "relmse_target": ev["target"], "relmse_eps": ld.LOSS_EPS,
        "time_to_target_ms": {"plain": plain_t, "eaw_tuned": eaw_t, "svgf": svgf_t, "learned": learned_t},
        "svgf_best_relmse": min(r["svgf"] for r in rows),
        "speedup_learned_vs_plain": (plain_t["ms"] / learned_t["ms"]) if learned_t["ms"] else None,
        "speedup_learned_vs_eaw": (eaw_t["ms"] / learned_t["ms"]) if (learned_t["ms"] and eaw_t["ms"]) else None,
        "speedup_learned_vs_eaw_median_over_seeds": statistics.median(speedups) if speedups else None,
        "per_seed": [{"seed": e["seed"], "time_to_target_ms": {k: e[k] for k in ("plain", "eaw_tuned", "svgf", "learned")},
                      "speedup_learned_vs_eaw": (e["eaw_tuned"]["ms"] / e["learned"]["ms"])
                      if (e["learned"]["ms"] and e["eaw_tuned"]["ms"]) else None} for e in scenes],
        "ms_per_frame": {"plain": ms_plain, "with_features": ms_feat, "feature_frames": kf},
        "denoise_ms": {"eaw": eaw_cost, "learned": net_cost},
        "svgf_ms_per_frame": svgf_cost,
        "curve": rows, "reference_render_s": ref_s,
        "training": {"data_s": data.seconds, "data_paths": data.paths, "train_s": hist["seconds"],
                     "loss_curve": hist["loss_curve"], "step_ms": step_ms, "launches_per_step": launches_per_step,
                     "conv_gflop_per_step": conv_flop / 1e9,
                     "roofline": {"bound": "tensor", "achieved": conv_flop / (step_ms / 1e3) / 1e12, "peak": peak,
                                  "unit": "TFLOP/s", "frac": conv_flop / (step_ms / 1e3) / 1e12 / peak,
                                  "note": f"convolution flops of a whole training step / step time; peak {peak_kind}"}},
    }
    return out


# NanoVDB sparse configuration: 2048x1024x1536 virtual voxels, 8^3 leaves with ~12% of the leaf
# slots active (seeded fBm cumulus, remap contrast 2, values below 0.85 empty), extinction 2000,
# 1920x1080, max 256 bounces; delta tracking through the sparse volume and HDDA decomposition
# tracking (the reference's sparse empty-space-skipping tracker), fp32 and fp16 leaf values.
SPARSE_DIMS = (2048, 1024, 1536)
SPARSE_RES = (1920, 1080)
SPARSE_SPP_PER_STEP = 128  # the configuration's 128 spp, one step = one full render
SPARSE_EXTINCTION = 2000.0
SPARSE_MAX_BOUNCES = 256
SPARSE_SEED = 3


def run_sparse(vpt, lib, ctx, stream, ctypes_stream, barrier, max_over_ranks, world, steps=2):
    import ctypes
    import torch

    t0 = time.perf_counter()
    vpt.set_max_grid_extent(0.5)
    _lib_check = vpt._lib.check
    _lib_check(lib.vpt_set_option(ctx, b"fbm_contrast", 2.0), "contrast", ctx)
    vpt.generate_fbm_cloud(SPARSE_DIMS, seed=SPARSE_SEED, threshold=0.85)
    _lib_check(lib.vpt_set_option(ctx, b"fbm_contrast", 3.5), "contrast", ctx)
    vpt.set_use_sparse_grid(True)
    info = vpt._sparse_info()
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    slots = np.prod([math.ceil(n / 8) for n in SPARSE_DIMS])
    vpt.set_extinction_scale(SPARSE_EXTINCTION)
    vpt.set_max_bounces(SPARSE_MAX_BOUNCES)
    w, h = SPARSE_RES
    img = torch.zeros((4, h, w), dtype=torch.float32, device="cuda")
    out = {"workload": f"NanoVDB-layout sparse grid {SPARSE_DIMS[0]}x{SPARSE_DIMS[1]}x{SPARSE_DIMS[2]} virtual voxels, "
                       f"{w}x{h}, {SPARSE_SPP_PER_STEP} spp/step, extinction {SPARSE_EXTINCTION:g}, "
                       f"max {SPARSE_MAX_BOUNCES} bounces",
           "leaves": int(info.leaves), "leaf_occupancy": float(info.leaves) / float(slots),
           "device_bytes": int(info.device_bytes), "build_s": build_s, "trackers": {}}
    for fp16 in (False, True):
        if fp16:
            vpt.set_sparse_grid_fp16(True)
            vpt.set_use_sparse_grid(True)
            out["device_bytes_fp16"] = int(vpt._sparse_info().device_bytes)
        for name, mode in (("delta", 0), ("decomposition_hdda", 3)):
            vpt.set_vpt_mode(mode)
            vpt.render_frame(img, 1)
            barrier()
            vpt.reset_stats()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                _lib_check(lib.vpt_render_frames(ctx, SPARSE_SPP_PER_STEP, ctypes_stream), "render", ctx)
            e1.record(stream)
            barrier()
            ms = max_over_ranks(e0.elapsed_time(e1))
            st = vpt.get_stats()
            key = name + ("_fp16" if fp16 else "")
            out["trackers"][key] = {"path_samples_per_s": w * h * SPARSE_SPP_PER_STEP * steps * world / (ms / 1e3),
                                    "lookups_per_path": st["density_lookups"] / max(1, st["paths"]),
                                    "lookups_per_s": st["density_lookups"] * world / (ms / 1e3),
                                    "ms_per_step": ms / steps}
    vpt.set_sparse_grid_fp16(False)
    vpt.set_use_sparse_grid(False)
    return out


# Batched configuration: 64 independent scenes in one persistent launch (captured CUDA graph,
# autotuned blocks per SM), delta tracking: grids log-uniform 64^3..512^3 (fBm, seed 1000 + i),
# extinction log-uniform 100..2000, g uniform 0.6..0.9, images log-uniform 128^2..1024^2, spp uniform
# 1..64, per-scene sun direction and camera pose.
BATCH_SCENES = 64


def batch_specs(n=None):
    n = n or BATCH_SCENES
    rng = np.random.default_rng(1000)
    specs = []
    for i in range(n):
        grid = int(round(math.exp(rng.uniform(math.log(64), math.log(512)))))
        res = int(round(math.exp(rng.uniform(math.log(128), math.log(1024)))))
        specs.append(dict(seed=1000 + i, grid=grid, res=res, spp=int(rng.integers(1, 65)),
                          extinction=float(math.exp(rng.uniform(math.log(100.0), math.log(2000.0)))),
                          g=float(rng.uniform(0.6, 0.9)), sun=sun_dir(1000 + i), cam=camera_pos(1000 + i)))
    return specs


def run_batch(lib, stream, ctypes_stream, barrier, max_over_ranks, world, steps=3):
    import ctypes
    import torch
    from cloudrendering_b200 import _lib
    from cloudrendering_b200.scene_sharding import assign_lpt, scene_cost

    all_specs = batch_specs()
    # several ranks: each renders its share of the scenes (longest processing time first by estimated
    # density lookups), no exchange; the aggregate rate is all scenes' paths over the slowest rank's time
    rank = int(os.environ.get("RANK", "0"))
    costs = [scene_cost(sp["res"], sp["res"], sp["spp"], sp["extinction"]) for sp in all_specs]
    mine = assign_lpt(costs, world)[rank]
    specs = [all_specs[i] for i in mine]
    paths_all = sum(sp["res"] * sp["res"] * sp["spp"] for sp in all_specs)
    ctxs = []
    t0 = time.perf_counter()
    best = ctypes.c_int()
    try:
        for sp in specs:
            c = ctypes.c_void_p()
            _lib.check(lib.vpt_create(ctypes.byref(c), torch.cuda.current_device()), "create")
            ctxs.append(c.value)
            h = ctxs[-1]

            def chk(st, what, h=h):
                _lib.check(st, what, h)

            chk(lib.vpt_set_max_grid_extent(h, 0.5), "extent")
            chk(lib.vpt_generate_fbm_grid(h, sp["grid"], sp["grid"], sp["grid"], sp["seed"], 6, 2.0, 0.5, 3.0, 0.3),
                "fbm")
            chk(lib.vpt_set_vpt_mode(h, 0), "mode")
            chk(lib.vpt_set_extinction_scale(h, sp["extinction"]), "extinction")
            chk(lib.vpt_set_scattering_albedo(h, _lib.farr([0.99] * 3)), "albedo")
            chk(lib.vpt_set_phase_g(h, sp["g"]), "g")
            chk(lib.vpt_set_builtin_environment_map(h, 3), "env")
            chk(lib.vpt_set_sky_color(h, _lib.farr([0.2] * 3)), "sky")
            chk(lib.vpt_set_sun(h, _lib.farr(sp["sun"]), _lib.farr([5.0] * 3)), "sun")
            chk(lib.vpt_set_camera(h, _lib.farr(sp["cam"]), _lib.farr([0, 0, 0]), _lib.farr([0, 1, 0]),
                                   math.radians(60.0), 1.0 / 512.0, 80.0), "camera")
            chk(lib.vpt_set_max_bounces(h, MAX_BOUNCES), "bounces")
            chk(lib.vpt_set_resolution(h, sp["res"], sp["res"]), "resolution")
            chk(lib.vpt_set_denoiser(h, 0), "denoiser")
        torch.cuda.synchronize()
        setup_s = time.perf_counter() - t0
        paths_per_step = sum(sp["res"] * sp["res"] * sp["spp"] for sp in specs)
        frames = (ctypes.c_int * len(specs))(*[sp["spp"] for sp in specs])
        arr = (ctypes.c_void_p * len(ctxs))(*ctxs)
        b = ctypes.c_void_p()
        _lib.check(lib.vpt_batch_create(ctypes.byref(b), arr, len(ctxs)), "batch")
        try:
            if lib.vpt_batch_autotune(b, frames, ctypes_stream, ctypes.byref(best)) != 0:
                raise RuntimeError(lib.vpt_batch_last_error(b).decode())
            if lib.vpt_batch_render(b, frames, ctypes_stream) != 0:  # captures the graph
                raise RuntimeError(lib.vpt_batch_last_error(b).decode())
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                if lib.vpt_batch_render(b, frames, ctypes_stream) != 0:
                    raise RuntimeError(lib.vpt_batch_last_error(b).decode())
            e1.record(stream)
            barrier()
            ms_batch = max_over_ranks(e0.elapsed_time(e1)) / steps
        finally:
            lib.vpt_batch_destroy(b)
        # the same frames as one launch per scene
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for c, sp in zip(ctxs, specs):
            _lib.check(lib.vpt_render_frames(c, sp["spp"], ctypes_stream), "render", c)
        e1.record(stream)
        barrier()
        ms_seq = max_over_ranks(e0.elapsed_time(e1))
    finally:
        for c in ctxs:
            lib.vpt_destroy(c)
    return {"workload": f"{len(all_specs)} independent scenes (grids 64^3..512^3, images 128^2..1024^2, 1..64 spp, "
                        "extinction 100..2000, g 0.6..0.9), delta tracking, one persistent launch per step "
                        "(CUDA graph, autotuned blocks per SM)"
                        + (f"; scenes sharded over {world} ranks by longest processing time" if world > 1 else ""),
            "scenes": len(all_specs), "scenes_on_rank0": len(specs), "paths_per_step": paths_all, "setup_s": setup_s,
            "autotuned_blocks_per_sm": best.value,
            "batched_path_samples_per_s": paths_all / (ms_batch / 1e3), "ms_per_step": ms_batch,
            "one_launch_per_scene_path_samples_per_s": paths_all / (ms_seq / 1e3)}


def cpu_baseline(lib, ctx, vpt, target_s=12.0):
    """CPU oracle on a band of rows of the same workload (1 spp), all host cores."""
    import ctypes
    from oracle import bridge

    n = GRID ** 3
    grid = np.empty((GRID, GRID, GRID), np.float32)
    _lib_check = vpt._lib.check
    _lib_check(lib.vpt_get_dense_grid(ctx, grid.ctypes.data_as(ctypes.c_void_p), 0), "get grid", ctx)
    inv = (ctypes.c_float * 16)()
    vp = (ctypes.c_float * 16)()
    vpt.set_vpt_mode_from_name("Delta Tracking")
    _lib_check(lib.vpt_get_camera_matrices(ctx, inv, vp), "camera", ctx)
    vmin, vmax = bridge.minmax(grid)
    dens = bridge.normalize(grid, vmin, vmax)
    bmin, bmax = bridge.grid_bounds(GRID, GRID, GRID, 0.5)
    f32 = np.float32
    vpu = [float(f32(GRID / (float(f32(b1)) - float(f32(b0))))) for b0, b1 in zip(bmin, bmax)]
    sd = np.array(sun_dir(SEED), np.float32)
    dl = np.sqrt(f32(f32(sd[0] * sd[0]) + f32(sd[1] * sd[1])) + f32(sd[2] * sd[2]), dtype=np.float32)
    sc = bridge.Scene(inv_view_proj=list(inv), width=RES, height=RES, frame_count=0, num_frames=1, seed_offset=0,
                      mode=0, interp=1, max_bounces=MAX_BOUNCES, use_ess=0, box_min=bmin, box_max=bmax, nx=GRID,
                      ny=GRID, nz=GRID, vox_per_unit=vpu,
                      border_density=float((f32(0.0) - f32(vmin)) / (f32(vmax) - f32(vmin))), extinction=EXTINCTION,
                      albedo=0.99,
                      g=0.85, env_kind=3, use_linear_rgb=1, env_image_linear=1,
                      sun_dir=[float(f32(sd[i] / dl)) for i in range(3)], sun_intensity=[5.0] * 3,
                      sky_color=[0.2] * 3, env_intensity=[1.0] * 3, density=dens)
    threads = os.cpu_count() or 1
    # the whole image (the GPU arm's pixel mix) at as many spp as fit in about target_s
    frames, elapsed, lookups = 1, 0.0, 0
    while True:
        sc.set("num_frames", frames)
        t0 = time.perf_counter()
        _, _, lookups = sc.render(threads)
        elapsed = time.perf_counter() - t0
        if elapsed >= target_s / 3 or frames >= 4096:
            break
        frames = min(4096, max(frames * 2, int(frames * target_s / max(elapsed, 1e-3))))
    paths = RES * RES * frames
    return {"value": paths / elapsed, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"delta tracking, the whole {RES}x{RES} image x {frames} spp ({paths} paths, {elapsed:.1f} s)",
            "lookups_per_s": lookups / elapsed, "lookups_per_path": lookups / paths}


def run_reference(args):
    """CPU reference arm: the oracle restatement of the reference shaders on this host's cores."""
    import ctypes
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import bridge
    grid = bridge.fbm(GRID, SEED, base_frequency=3.0, contrast=3.5)
    vmin, vmax = bridge.minmax(grid)
    dens = bridge.normalize(grid, vmin, vmax)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from tests.harness import SceneSpec, camera_inv_view_proj
    sp = SceneSpec(cam_pos=camera_pos(SEED), fovy=math.radians(60.0), near=1.0 / 512.0, far=80.0, width=RES,
                   height=RES)
    inv = camera_inv_view_proj(sp)
    bmin, bmax = bridge.grid_bounds(GRID, GRID, GRID, 0.5)
    f32 = np.float32
    vpu = [float(f32(GRID / (float(f32(b1)) - float(f32(b0))))) for b0, b1 in zip(bmin, bmax)]
    sd = np.array(sun_dir(SEED), np.float32)
    sd = sd / np.linalg.norm(sd)
    sc = bridge.Scene(inv_view_proj=inv, width=RES, height=RES, frame_count=0, num_frames=1, seed_offset=0, mode=0,
                      interp=1, max_bounces=MAX_BOUNCES, use_ess=0, box_min=bmin, box_max=bmax, nx=GRID, ny=GRID,
                      nz=GRID, vox_per_unit=vpu, border_density=0.0, extinction=EXTINCTION, albedo=0.99, g=0.85,
                      env_kind=3, use_linear_rgb=1, env_image_linear=1, sun_dir=sd.tolist(), sun_intensity=[5.0] * 3,
                      sky_color=[0.2] * 3, env_intensity=[1.0] * 3, density=dens)
    threads = os.cpu_count() or 1
    # each step: the whole image at 1 spp (the GPU arm's pixel mix), frame index = step
    sc.set("num_frames", 1)
    for i in range(args.warmup):
        sc.set("frame_count", 1000 + i)
        sc.render_rows(RES // 2 - 4, RES // 2 + 4, threads)
    times = []
    lookups = 0
    for i in range(args.steps):
        sc.set("frame_count", i)
        t0 = time.perf_counter()
        _, _, lk = sc.render(threads)
        times.append(time.perf_counter() - t0)
        lookups += lk
    total = sum(times)
    paths = RES * RES * args.steps
    value = paths / total
    sample = f"delta tracking, the whole {RES}x{RES} image at 1 spp per step, {threads} threads"
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total / args.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded fBm Perlin cloud)", "config": workload_config(world),
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "lookups_per_s": lookups / total, "lookups_per_path": lookups / paths,
    }), flush=True)


def profile_trace(spp):
    """Two launches of the delta tracker on the bench scene (1 frame, then `spp` frames) for ncu:
    `ncu -k regex:trace_refill -s 1 -c 1 ... python bench.py --profile-trace SPP` captures the second."""
    import torch
    from cloudrendering_b200 import vpt, _lib
    torch.cuda.set_device(0)
    lib = _lib.load()
    vpt.initialize()
    ctx = vpt.context_handle()
    setup_scene(vpt, 0)
    _lib.check(lib.vpt_set_option(ctx, b"density_texture", float(DENSITY_TEXTURE)), "density_texture", ctx)
    _lib.check(lib.vpt_set_option(ctx, b"refill_min_lanes", float(REFILL_MIN_LANES)), "refill_min_lanes", ctx)
    vpt.set_vpt_mode_from_name("Delta Tracking")
    _lib.check(lib.vpt_set_resolution(ctx, RES, RES), "resolution", ctx)
    cs = __import__("ctypes").c_void_p(torch.cuda.current_stream().cuda_stream)
    for frames in (1, spp):
        _lib.check(lib.vpt_synchronize(ctx, cs), "sync", ctx)
        vpt.reset_stats()
        _lib.check(lib.vpt_render_frames(ctx, frames, cs), "render", ctx)
    _lib.check(lib.vpt_synchronize(ctx, cs), "sync", ctx)
    st = vpt.get_stats()
    print(json.dumps({"profile_trace": {"grid": GRID, "image": RES, "spp": spp, "paths": st["paths"],
                                        "density_lookups": st["density_lookups"]}}), flush=True)
    vpt.cleanup()


def main():
    global DENSITY_TEXTURE
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-sparse", action="store_true", help="skip the NanoVDB sparse configuration")
    ap.add_argument("--no-batch", action="store_true", help="skip the 64-scene batched configuration")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-denoiser configuration")
    ap.add_argument("--profile-trace", type=int, default=0, metavar="SPP",
                    help="profiling entry: set up the bench scene, render one warm-up frame, then one launch of "
                         "SPP frames of delta tracking, and exit (capture the second trace launch with ncu)")
    ap.add_argument("--streaming", action="store_true",
                    help="run only the streaming-kernel leg (builders, EAW, KPN apply) and print its JSON")
    ap.add_argument("--density-texture", type=int, choices=[0, 1], default=None,
                    help="delta tracking's density fetch: 1 = the grid's 3D texture object, 0 = global loads "
                         f"(default {DENSITY_TEXTURE})")
    ap.add_argument("--workload", choices=["full", "small"], default="full",
                    help="small: 384^3 grid, 512^2, 4 spp/step (for ncu captures; not a bench line)")
    args = ap.parse_args()
    if args.density_texture is not None:
        DENSITY_TEXTURE = args.density_texture
    if args.warmup < 3:
        args.warmup = 3
    if args.workload == "small":
        global GRID, RES, SPP_PER_STEP
        GRID, RES, SPP_PER_STEP = 384, 512, 4
        args.no_cpu_baseline = True
        global SPARSE_DIMS, SPARSE_RES, BATCH_SCENES
        SPARSE_DIMS, SPARSE_RES = (512, 256, 384), (480, 270)
        BATCH_SCENES = 8
    if args.streaming:
        import torch
        from cloudrendering_b200 import _lib
        torch.cuda.set_device(0)
        print(json.dumps({"streaming_kernels": run_streaming(_lib.load(), torch.cuda.current_stream())}), flush=True)
    elif args.profile_trace:
        profile_trace(args.profile_trace)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
