"""Benchmark: fit iterations per second (forward + backward + Adam) of the
inverse-rendering fit at 1024^2 with a batch of 16 views -- UV sphere
256x128 (65,024 triangles) displaced N(0,0.02), 16 views of 1024x1024 at
seeded cameras, 2048^2 RGBA texture with 12 mip levels, 32 SG lobes, Adam
on positions, texture and lobes -- with seeded synthetic inputs (no
dataset).  The fused graph-captured step ("batched") is timed beside the
plain one-launch-per-operator pipeline.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl vcl|reference]
                  [--views V] [--config config1|config2|config5|mix|serve]

One JSON line on rank 0.  Multi-GPU runs are independent replicas (one fit
job per GPU, no data-path collective; weak scaling); times are max over
ranks.  See the module-level notes at each measured quantity.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+bwd+Adam iters/s @1024² batch 16, batched vs plain; p50/p99 fit-job latency"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="vcl", choices=["vcl", "reference"])
    ap.add_argument("--views", type=int, default=None, help="views per iteration (default: 16, config5: 4)")
    ap.add_argument("--config", default="config2", choices=["config1", "config2", "config5", "mix", "serve"])
    ap.add_argument("--scenes", type=int, default=64, help="mix: scenes per batched launch")
    ap.add_argument("--jobs", type=int, default=32, help="serve: fit jobs submitted")
    ap.add_argument("--lams", default="10,30,100,300,1000", help="serve: arrival rates (jobs/s)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mix", action="store_true", help="default run: skip the batched-vs-plain mix measurement")
    ap.add_argument("--no-serve", action="store_true", help="default run: skip the serving measurement")
    ap.add_argument("--no-config5", action="store_true",
                    help="default run: skip the dense-stress fit iteration (4 x 2048^2, 1.31M triangles, 4096^2 texture)")
    ap.add_argument("--serve-lam", type=float, default=100.0, help="default run: serving arrival rate (jobs/s)")
    ap.add_argument("--serve-jobs", type=int, default=24, help="default run: serving jobs per repeat")
    ap.add_argument("--serve-repeats", type=int, default=3, help="default run: serving repeats")
    ap.add_argument("--no-stages", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--strategy", default="both", choices=["both", "plain", "fused"])
    ap.add_argument("--raster-schedule", default="tuned", choices=["tuned", "size"],
                    help="fit jobs time raster schedules (tuned) or take the size-based one (size; "
                         "deterministic, e.g. under a profiler)")
    return ap.parse_args()


def make_scene(args):
    from vcl_b200 import scenes
    if args.config == "config1":
        return scenes.config1()
    if args.config == "config5":
        return scenes.config5(views=args.views or 4)
    return scenes.config2(views=args.views or 16)


def bench_config(S, world):
    """The `config` object of both arms' JSON lines (same workload, same keys)."""
    return {"workload": workload_name(S), "global_batch": S.views * world, "seq_len": 0,
            "parallelism": f"replicas x{world}",
            "adam": {"lr": S.lr, "lr_pos": S.lr_pos or S.lr, "betas": [0.9, 0.999], "eps": 1e-8},
            "l2": "per-step working set > 2 GB (larger than the 126 MB L2); no flush"}


def workload_name(S):
    return (f"fit iteration: {S.name}: {S.nt} tris, {S.views} views {S.W}x{S.H}, texture {S.tex_w}^2x{S.C} "
            f"({S.levels} levels), {S.K} SG lobes, Adam on positions+texture+lobes")


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples during the timed region (clock, throttle reasons).
    Started before the warm-up (so that nvidia-smi is running when timing
    begins), sampling every 20 ms; window(t0, t1) keeps the samples whose host
    arrival time falls inside the timed region (the first later sample when a
    short region caught none)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None
        self.win = None

    def window(self, t0, t1):
        self.win = (t0, t1)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append((time.perf_counter(), [x.strip() for x in line.split(",")]))

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        rows = [r for _, r in self.rows]
        if self.win is not None:
            t0, t1 = self.win
            inside = [r for t, r in self.rows if t0 <= t <= t1]
            later = [r for t, r in self.rows if t > t1][:1]
            rows = inside or later
        self.rows = rows
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) >= 9:
                for n, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# ------------------------------------------------------------ algorithmic bytes
def stage_bytes(S, ncov):
    """Compulsory FP32 traffic per fit iteration by stage (caches ignored,
    each buffer counted once).  Every per-pixel kernel reads the raster word
    of all N pixels; the other per-pixel inputs are read only at the ncov
    covered pixels (background pixels return early), and outputs are
    written at all N pixels where the kernel clears the background, at the
    covered ones where it does not."""
    N = S.W * S.H * S.views
    C = S.C
    ntex = S.tex_w * S.tex_h
    npyr_bytes = ntex * C * 4 * 4 / 3
    texel_fwd = min(npyr_bytes, ncov * 8 * C * 4)
    return {
        "raster_fwd": S.nv * 16 * S.views + S.nt * 12 + N * 32,
        "interp_fwd": N * 16 + ncov * 16 + N * (8 + 16),                 # rast; db; uv + DA written everywhere
        "texture_fwd": N * 16 + ncov * (8 + 16) + N * C * 4 + texel_fwd,  # rast; uv, DA; colour everywhere
        "normal_axis": N * 16 + N * 12,
        "view_axis": N * 12,
        "sg_specular_fwd": N * 16 + ncov * (12 + 12 + 4) + N * 20,        # rast; n, view, roughness; 3 outputs
        "sg_fwd": N * 16 + ncov * (12 + C * 4 + 12 + 8) + N * C * 4 + S.K * (4 + C) * 4,
        "antialias_fwd": N * (16 + C * 4) + N * C * 4,
        "mse": N * C * 4 * 2 + N * C * 4,
        "antialias_bwd": N * (C * 8 + 16) + N * C * 4,
        "sg_bwd": N * 16 + ncov * (C * 4 * 2 + 12 + 12 + 8) + ncov * C * 4,
        "texture_bwd": N * 16 + ncov * (C * 4 + 8 + 16) + ncov * 8 + texel_fwd,
        "interp_bwd": N * 16 + ncov * 8 + ncov * 8,
        "raster_bwd": N * 16 + ncov * 8,
        "project": S.nv * 12 * 2,
        "optimizer": 28 * (ntex * C + S.nv * 3 + S.K * (4 + C)) + ntex * C * 4 * (1 / 3 + 2 / 3 + 1 + 4 / 3),
    }


def fused_bytes(S, ncov):
    """Compulsory FP32 traffic of each fused-step stage (one launch; caches
    ignored, each buffer counted once).  N = views*W*H pixels, ncov of them
    covered, C = 4; inputs other than the raster word are read at covered
    pixels only."""
    N = S.W * S.H * S.views
    ntex = S.tex_w * S.tex_h
    texels = min(ntex * 16 * 4 / 3, ncov * 8 * 16)      # trilinear reads, at most the pyramid once
    verts = S.views * S.nv * 16
    return {
        "raster": verts + S.nt * 12 + N * 32,                       # clip, indices -> rast + db
        # rast (all), db (covered) -> colour, diffuse env (all), shading records (covered)
        "shade_fwd": N * 16 + ncov * 16 + S.nv * 20 + texels + N * 32 + ncov * 52,
        "aa_fwd_mse": N * 64 + verts,                               # rast, colour, target -> image gradient, loss
        "aa_bwd": N * 64 + verts * 2,                               # rast, colour, grad -> colour grad, clip grad
        "bwd_pix": N * 16 + ncov * 48 + texels + verts * 2,         # rast; db, colour grad, diffuse env -> texel, clip grads
        "sg_lobes": ncov * (52 + 16) + S.K * 32,                    # shading records, colour grad -> lobe grads
    }


# DRAM bytes per pixel of the fused step's two largest kernels, from one ncu
# capture (dram__bytes_read.sum + dram__bytes_write.sum of one launch on 4
# views of 1024x1024 of this workload, divided by the pixels); their traffic
# grows with the pixel count.
DRAM_BYTES_PER_PIXEL = {
    "bwd_pix": (321.2e6 + 64.6e6) / (4 * 1024 * 1024),
    "sg_lobes": (182.8e6 + 4.0e6) / (4 * 1024 * 1024),
}
# What bounds each of them instead of HBM bandwidth (same capture).
BOUND_NOTE = {
    "bwd_pix": "k_bwd_pix is bound by the scatter of texel gradients through L2 (vector reductions; "
               "L2 ~50% busy, warps waiting on loads and the LSU queue), not by HBM bandwidth",
    "sg_lobes": "k_sg_lobes is bound by its FMA pipe and MUFU (per pixel and lobe: 2 rsqrt, 4 ex2 and ~65 FP32 "
                "operations issued as ~33 paired instructions for two pixels), not by HBM",
}


# ------------------------------------------------------------ measured peaks
def measure_unit_peaks(ctx, stream, reps=3):
    """Peak rates of the L2 vector reductions and of the MUFU pipe on this
    GPU, from the library's throughput probes (best of `reps`, CUDA events on
    the launching stream): red.global.add.v4.f32 per second over a 32 MB
    buffer (inside L2), and ex2/rsqrt operations per second."""
    import ctypes
    import torch
    from vcl_b200 import capi
    L = capi.lib()
    sh = stream.cuda_stream
    buf = torch.zeros(8 << 20, dtype=torch.float32, device="cuda")
    out = torch.zeros(L.vcl_probe_mufu_threads(ctx.h), dtype=torch.float32, device="cuda")
    n = ctypes.c_longlong()

    def best(fn):
        fn()
        t = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            stream.synchronize()
            t.append(e0.elapsed_time(e1) * 1e-3)
        return min(t)

    t_red = best(lambda: ctx._check(L.vcl_probe_red_throughput(ctx.h, buf.data_ptr(), buf.numel(), 20,
                                                               ctypes.byref(n), sh), "probe"))
    reds = n.value
    t_mufu = best(lambda: ctx._check(L.vcl_probe_mufu_throughput(ctx.h, out.data_ptr(), 4096, ctypes.byref(n), sh),
                                     "probe"))
    mufu = n.value
    t_fma = best(lambda: ctx._check(L.vcl_probe_fma_throughput(ctx.h, out.data_ptr(), 16384, ctypes.byref(n), sh),
                                    "probe"))
    fma = n.value
    return {"l2_red_v4_per_s": reds / t_red, "mufu_ops_per_s": mufu / t_mufu, "fma_ops_per_s": fma / t_fma,
            "how": "vcl_probe_red_throughput (coalesced red.global.add.v4.f32 over 32 MB, 20 passes), "
                   "vcl_probe_mufu_throughput (8 independent ex2.approx/rsqrt.approx chains per thread) and "
                   "vcl_probe_fma_throughput (8 independent paired-FP32 fma chains per thread), 8 blocks of 256 "
                   "per SM; best of 3, CUDA events"}


# ------------------------------------------------------------------ vcl arm
def run_vcl(args, rank, world):
    import torch
    from vcl_b200 import capi, replicas

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    S = make_scene(args)
    ctx = capi.Context(dev)
    if args.raster_schedule == "size":
        ctx.set_raster_autotune(0)
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    N = S.W * S.H * S.views
    img_numel = N * S.C

    # targets: the true scene rendered once + N(0, 0.05) pixel noise
    truth = capi.Fit(ctx, S, tex=S.tex_target, pos=S.pos_target,
                     lobes=(S.lobe_axis, S.lobe_sharp, S.lobe_amp), learn=(0, 0, 0))
    target = torch.zeros(img_numel, dtype=torch.float32, device="cuda")
    with torch.cuda.stream(stream):
        truth.render(target, sh)
        g = torch.Generator(device="cuda").manual_seed(S.seed + 1)
        target.add_(torch.randn(img_numel, generator=g, device="cuda") * S.noise)
    stream.synchronize()
    truth.close()

    def make_fit(strategy):
        f = capi.Fit(ctx, S, strategy=strategy)
        f.set_target(target, sh, is_device=True)
        return f

    def timed(fit, steps, warmup, sampler=None):
        for _ in range(warmup):
            fit.step(sh)
        stream.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        for _ in range(steps):
            fit.step(sh)
        e1.record(stream)
        stream.synchronize()
        if sampler is not None:
            sampler.window(t0, time.perf_counter())
        barrier()
        return e0.elapsed_time(e1)

    def barrier():
        torch.cuda.synchronize()
        replicas.barrier()
        torch.cuda.synchronize()

    maxr = replicas.max_over_ranks

    out = {}
    strategies = [] if args.strategy == "fused" else [("plain", capi.FIT_PLAIN)]
    if args.strategy != "plain":
        strategies.append(("fused", capi.FIT_FUSED))
    clocks = ClockSampler(dev)
    results = {}
    launches = {}
    losses = {}
    for name, strat in strategies:
        fit = make_fit(strat)
        if name == strategies[-1][0]:
            clocks.start()
        ms = maxr(timed(fit, args.steps, args.warmup, clocks if name == strategies[-1][0] else None))
        if name == strategies[-1][0]:
            clk = clocks.stop()
        results[name] = ms
        launches[name] = fit.launches_per_step()
        losses[name] = fit.read_loss(sh)
        if strat == capi.FIT_FUSED:
            out["raster_tuning"] = fit.raster_tuning()
            out["fused_kernel_ms"] = fit.time_kernels(sh, reps=3)   # after the timed region
        fit.close()
    best = strategies[-1][0]
    ms_per_step = results[best] / args.steps
    value = world * 1000.0 / ms_per_step

    out.update(results=results, launches=launches, losses=losses, value=value, ms_per_step=ms_per_step,
               clocks=clk, scene=S, best=best, e2e_ms=None)
    if args.no_e2e:
        if rank == 0 and not args.no_stages:
            out["stages"] = stage_times(ctx, S, target, stream)
        ctx.close()
        return out
    # end to end through the public API: every step's target images and
    # cameras go host -> device (pinned), the loss comes back device -> host.
    # The target of step i+1 is staged on a copy stream while step i runs.
    fit = make_fit(strategies[-1][1])
    host_target = torch.empty(img_numel, dtype=torch.float32, pin_memory=True)
    host_target.copy_(target.cpu())
    host_mvp = torch.from_numpy(np.ascontiguousarray(S.mvp, dtype=np.float32)).pin_memory()
    host_pvinv = torch.from_numpy(np.ascontiguousarray(S.pvinv, dtype=np.float32)).pin_memory()
    copy_stream = torch.cuda.Stream()
    cs = copy_stream.cuda_stream

    host_losses = torch.zeros(max(args.steps, args.warmup, 1), dtype=torch.float32).pin_memory()

    def e2e_run(n, e0=None, e1=None):
        if e0 is not None:
            e0.record(copy_stream)
        fit.stage_target(host_target, cs)
        for i in range(n):
            fit.set_cameras(host_mvp, host_pvinv, sh)
            fit.step(sh)
            if i + 1 < n:
                fit.stage_target(host_target, cs)
            # device->host read of every step's loss into pinned memory, queued
            # behind the step (the host runs ahead; all reads land before e1)
            fit.read_loss_async(host_losses.data_ptr() + 4 * i, sh)
        if e1 is not None:
            e1.record(stream)

    e2e_run(args.warmup)
    stream.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_run(args.steps, e0, e1)
    stream.synchronize()
    copy_stream.synchronize()
    barrier()
    e2e_ms = maxr(e0.elapsed_time(e1)) / args.steps
    e2e_losses = host_losses[:args.steps].numpy().copy()
    if not np.all(np.isfinite(e2e_losses)) or not np.all(e2e_losses > 0):
        raise RuntimeError(f"end-to-end loop read back invalid losses: {e2e_losses[:4]} ...")

    # the same loop with the target images resident (uploaded once, as the
    # reference's preset renders its targets on the device): per step only
    # the cameras go host -> device and the loss comes back
    def cam_run(n, e0=None, e1=None):
        if e0 is not None:
            e0.record(stream)
        for i in range(n):
            fit.set_cameras(host_mvp, host_pvinv, sh)
            fit.step(sh)
            fit.read_loss_async(host_losses.data_ptr() + 4 * i, sh)
        if e1 is not None:
            e1.record(stream)

    fit.set_target(host_target, sh, is_device=False)
    cam_run(args.warmup)
    stream.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    cam_run(args.steps, e0, e1)
    stream.synchronize()
    barrier()
    out["e2e_resident_ms"] = maxr(e0.elapsed_time(e1)) / args.steps
    fit.close()

    out.update(results=results, launches=launches, losses=losses, value=value, ms_per_step=ms_per_step,
               e2e_ms=e2e_ms, clocks=clk, scene=S, best=best)
    if rank == 0 and not args.no_stages:
        out["stages"] = stage_times(ctx, S, target, stream)
    if rank == 0:
        out["unit_peaks"] = measure_unit_peaks(ctx, stream)
    ctx.close()
    return out


def stage_times(ctx, S, target, stream, reps=5):
    """Average device time of each operator of the plain pipeline on this
    workload (CUDA events on the launching stream around `reps` launches of
    that operator, after one untimed pass)."""
    import torch
    from vcl_b200 import capi
    sh = stream.cuda_stream
    W, H, V, C, K = S.W, S.H, S.views, S.C, S.K
    N = W * H * V
    f32 = lambda *s: torch.zeros(*s, dtype=torch.float32, device="cuda")
    dv = lambda a, dt=None: torch.from_numpy(np.ascontiguousarray(a if dt is None else a.astype(dt))).cuda()
    tri = dv(S.tri, np.int32)
    mvp, pos, uvattr, rot, nrm, pvinv = dv(S.mvp), dv(S.pos), dv(S.uv), dv(S.rot), dv(S.normal), dv(S.pvinv)
    axis, sharp, amp = dv(S.lobe_axis_init), dv(S.lobe_sharp_init), dv(S.lobe_amp_init)
    npyr = sum((S.tex_w >> l) * (S.tex_h >> l) * C for l in range(S.levels))
    pyr = f32(npyr)
    pyr[: S.tex_w * S.tex_h * C] = dv(S.tex_target).reshape(-1)
    clip, rast, db = f32(V, S.nv, 4), f32(N, 4), f32(N, 4)
    uv, uv_da, diffuse, normal, view = f32(N, 2), f32(N, 4), f32(N, C), f32(N, 3), f32(N, 3)
    rough = torch.full((N,), S.roughness, dtype=torch.float32, device="cuda")
    sax, ssh, sam, color, aa = f32(N, 3), f32(N), f32(N), f32(N, C), f32(N, C)
    g_aa, g_color, g_clip, loss = f32(N, C), f32(N, C), f32(V, S.nv, 4), f32(1)
    g_diff, g_axis, g_sharp, g_amp = f32(N, C), f32(K, 3), f32(K), f32(K, C)
    g_pyr, g_uv, g_bary, g_pos = f32(npyr), f32(N, 2), f32(N, 2), f32(S.nv, 3)
    n0 = S.tex_w * S.tex_h * C
    m, v = f32(n0), f32(n0)
    ops = [
        ("project", lambda: ctx.project_fwd(mvp, V, pos, S.nv, 4, clip, sh)),
        ("raster_fwd", lambda: ctx.rasterize_fwd(clip, S.nv, tri, S.nt, W, H, V, rast, db, sh)),
        ("interp_fwd", lambda: ctx.interpolate_fwd(rast, db, W, H, V, uvattr, S.nv, 2, tri, S.nt, uv, uv_da, sh)),
        ("texture_fwd", lambda: ctx.texture_fwd(rast, uv, uv_da, W, H, V, pyr, S.tex_w, S.tex_h, C, S.levels, diffuse, sh)),
        ("normal_axis", lambda: ctx.normal_axis_fwd(rast, W, H, V, rot, nrm, S.nv, tri, S.nt, normal, sh)),
        ("view_axis", lambda: ctx.view_axis_fwd(W, H, V, pvinv, view, sh)),
        ("sg_specular_fwd", lambda: ctx.sg_specular_fwd(rast, W, H, V, normal, view, rough, S.ior, sax, ssh, sam, sh)),
        ("sg_fwd", lambda: ctx.sg_fwd(rast, W, H, V, C, K, axis, sharp, amp, normal, diffuse, sax, ssh, sam, color,
                                      None, None, sh)),
        ("antialias_fwd", lambda: ctx.antialias_fwd(clip, S.nv, tri, S.nt, rast, W, H, V, C, color, aa, sh)),
        ("mse", lambda: ctx.mse(aa, target, N * C, g_aa, loss, sh)),
        ("antialias_bwd", lambda: ctx.antialias_bwd(clip, S.nv, tri, S.nt, rast, W, H, V, C, color, g_aa, g_color,
                                                    g_clip, sh)),
        ("sg_bwd", lambda: ctx.sg_bwd(rast, W, H, V, C, K, axis, sharp, amp, normal, diffuse, sax, ssh, sam, g_color,
                                      g_diff, g_axis, g_sharp, g_amp, None, None, None, sh)),
        ("texture_bwd", lambda: ctx.texture_bwd(rast, uv, uv_da, W, H, V, pyr, S.tex_w, S.tex_h, C, S.levels, g_diff,
                                                g_pyr, g_uv, None, sh)),
        ("interp_bwd", lambda: ctx.interpolate_bwd(rast, W, H, V, uvattr, S.nv, 2, tri, S.nt, g_uv, None, g_bary, sh)),
        ("raster_bwd", lambda: ctx.rasterize_bwd(clip, S.nv, tri, S.nt, W, H, V, rast, g_bary, g_clip, sh)),
        ("optimizer", lambda: ctx.adam_step(pyr, g_pyr, m, v, n0, 1e-2, 0.9, 0.999, 1e-8, 1, sh)),
    ]
    res = {}
    with torch.cuda.stream(stream):
        for name, fn in ops:
            fn()
        stream.synchronize()
        ncov = int((rast[:, 3] > 0).sum().item())
        for name, fn in ops:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                fn()
            e1.record(stream)
            stream.synchronize()
            res[name] = e0.elapsed_time(e1) / reps
        # GL tie census of this raster: pixels where a GL driver may legally
        # pick another triangle (centre exactly on an edge; equal depth)
        ctx.rasterize_fwd(clip, S.nv, tri, S.nt, W, H, V, rast, db, sh)
        flags = torch.zeros(N, dtype=torch.int32, device="cuda")
        counts = torch.zeros(2, dtype=torch.int64, device="cuda")
        ctx.raster_ties(clip, S.nv, tri, S.nt, W, H, V, rast, flags, counts, sh)
        stream.synchronize()
        c = counts.cpu().tolist()
    ties = {"edge_tie_pixels": c[0], "depth_tie_pixels": c[1], "covered_pixels": ncov, "pixels": N,
            "geometry": "the workload's starting positions"}
    return {"ms": res, "ncov": ncov, "ties": ties}


# ------------------------------------------------------------ CPU baseline
class RefStepper:
    """The reference's own CPU implementation of the path (oracle/_ref: its
    kernel sources compiled for the host, run with `threads` host threads;
    the raster stage is the CPU restatement of its GL rasterizer), stepped
    in bounded samples of one fit iteration: step s processes view s mod V
    -- project, raster, interpolate, texture, the four shading operators,
    antialias, MSE and every backward pass -- plus 1/V of the iteration's
    parameter work (Adam on a 1/V slice of texture level 0; on the last
    view also the mip gradient push-down, Adam on positions and lobes and
    the mip rebuild).  V consecutive steps are exactly one fit iteration of
    the workload, so iterations/s = steps / V / seconds."""

    def __init__(self, S, threads):
        from oracle import oracle as O
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import chain
        import types
        self.O, self.chain, self.S = O, chain, S
        lib = O.ref()
        self.kind = "reference"
        if lib is None:
            lib, self.kind = O.orc(), "port"
            self.threads = 1
        else:
            lib.set_threads(threads)
            self.threads = threads
        self.lib = lib
        self.views = []
        for v in range(S.views):
            sub = types.SimpleNamespace(**{k: getattr(S, k) for k in S.__dataclass_fields__})
            sub.views = 1
            sub.mvp = S.mvp[v:v + 1].copy()
            sub.pvinv = S.pvinv[v:v + 1].copy()
            sub.nv, sub.nt = S.nv, S.nt
            self.views.append(sub)
        rng = np.random.default_rng(S.seed + 11)
        self.targets = [rng.random((S.W * S.H, S.C), dtype=np.float32) for _ in range(S.views)]
        self.pyr = chain.build_pyramid(S, S.tex_init)
        self.pos = S.pos.copy()
        self.lobes = np.concatenate([S.lobe_axis_init.reshape(-1), S.lobe_sharp_init.reshape(-1),
                                     S.lobe_amp_init.reshape(-1)]).astype(np.float32)
        n0 = S.tex_w * S.tex_h * S.C
        z = lambda n: np.zeros(n, np.float32)
        self.n0 = n0
        self.mt, self.vt = z(n0), z(n0)
        self.mp, self.vp = z(self.pos.size), z(self.pos.size)
        self.ml, self.vl = z(self.lobes.size), z(self.lobes.size)
        self.s = 0

    def step(self):
        S, O, lib = self.S, self.O, self.lib
        V, K, C = S.views, S.K, S.C
        j = self.s % V
        t = self.s // V + 1
        ax = np.ascontiguousarray(self.lobes[:3 * K].reshape(K, 3))
        sh = np.ascontiguousarray(self.lobes[3 * K:4 * K])
        am = np.ascontiguousarray(self.lobes[4 * K:].reshape(K, C))
        r = self.chain.run_chain(lib, self.views[j], 0, target=self.targets[j], pos=self.pos, pyr=self.pyr,
                                 lobes=(ax, sh, am), raster_lib=O.orc(), adam_step=0)
        g = r["g_pyr"]
        if j == V - 1:
            lib_m = O.orc()
            lib_m.mip_pushdown(0, S.tex_w, S.tex_h, C, S.levels, g)
        a, b = self.n0 * j // V, self.n0 * (j + 1) // V
        p0 = self.pyr[a:b]
        lib.adam(0, b - a, p0, np.ascontiguousarray(g[a:b]), self.mt[a:b], self.vt[a:b], S.lr, 0.9, 0.999, 1e-8, t)
        if j == V - 1:
            O.orc().clamp(self.n0, self.pyr, 0.0, 1.0)
            O.orc().mip_build(S.tex_w, S.tex_h, C, S.levels, self.pyr)
            pp = self.pos.reshape(-1)
            lib.adam(0, pp.size, pp, np.ascontiguousarray(r["g_pos"].reshape(-1)), self.mp, self.vp,
                     S.lr_pos or S.lr, 0.9, 0.999, 1e-8, t)
            gl = np.concatenate([r["g_axis"].reshape(-1), r["g_sharp"].reshape(-1),
                                 r["g_amp"].reshape(-1)]).astype(np.float32)
            lib.adam(0, self.lobes.size, self.lobes, gl, self.ml, self.vl, S.lr, 0.9, 0.999, 1e-8, t)
        self.s += 1

    def close(self):
        if self.kind == "reference":
            self.lib.set_threads(1)

    def sample(self, steps):
        V = self.S.views
        return (f"{steps} steps of one view each ({steps / V:g} fit iterations of {V} views): every per-pixel "
                f"operator fwd+bwd through the reference's kernels for the host, raster by the CPU restatement "
                f"of its GL rasterizer, 1/{V} of texture Adam per step; mip push-down/rebuild and Adam on "
                f"positions and lobes once per {V} steps")


def time_reference(S, threads, steps, warmup):
    """(seconds per full fit iteration, kind, cores, sample) of the reference's
    CPU implementation over `steps` view-steps after `warmup` view-steps."""
    rs = RefStepper(S, threads)
    try:
        for _ in range(warmup):
            rs.step()
        t0 = time.perf_counter()
        for _ in range(steps):
            rs.step()
        dt = time.perf_counter() - t0
    finally:
        rs.close()
    return dt * S.views / steps, dt / steps, rs.kind, rs.threads, rs.sample(steps)


def run_reference(args, rank, world):
    """--impl reference: the reference's own CPU implementation of the path,
    all host threads, on the same workload, `--warmup` + `--steps` steps of
    one view (and 1/V of the parameter work) each."""
    S = make_scene(args)
    threads = os.cpu_count() or 1
    per_iter, per_step, kind, cores, sample = time_reference(S, threads, args.steps, args.warmup)
    v = 1.0 / per_iter
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": "iters/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step * 1000, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded; no dataset)",
            "config": bench_config(S, world),
            "step": f"one view of the {S.views}-view fit iteration + 1/{S.views} of its parameter work; "
                    f"{S.views} steps = one iteration",
            "cpu_baseline": {"value": v, "unit": "iters/s", "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": v, "unit": "iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_mixed(args, rank, world):
    """--config mix / serve: the batched engine and the serving loop on the
    uneven scene mix (one GPU; replicas when launched with several ranks)."""
    import torch
    from vcl_b200 import capi, mixbench
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    ctx = capi.Context(dev)
    clocks = ClockSampler(dev)
    clocks.start()
    if args.config == "mix":
        r = mixbench.run_mix(ctx, args.scenes, args.steps, args.warmup)
        metric = "scene fit-iterations/s (fwd+bwd+Adam), uneven scene mix, batched vs plain"
    else:
        r = mixbench.run_serve(ctx, args.jobs, [float(x) for x in args.lams.split(",")])
        metric = "fit-job p50/p99 latency and iters/s under Poisson arrivals, served vs plain one at a time"
    clk = clocks.stop()
    ctx.close()
    if rank != 0:
        return
    line = {"metric": metric, "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "dtype": "f32",
            "data": "synthetic (seeded; no dataset)", "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "clocks": clk}
    line.update(r)
    if args.config == "serve":
        best = max(r["sweep"], key=lambda x: x["iters_per_s"])
        line.update(value=best["iters_per_s"], unit="iters/s",
                    config={"workload": f"{r['jobs']} fit jobs from the uneven scene mix, U[50,500] iterations, "
                                        f"Poisson arrivals, {r['budget_gb']} GB admission budget"})
    print(json.dumps(line), flush=True)


def spawn_ranks(n):
    """`--gpus N` outside torchrun: start the N ranks through
    torch.distributed.run on this node and return its exit status."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def mix_summary(args):
    """Batched vs plain on the uneven 64-scene mix: one batched graph launch
    per iteration of every scene against the same scenes stepped one at a
    time through the plain pipeline (scene fit-iterations/s)."""
    import torch
    from vcl_b200 import capi, mixbench
    ctx = capi.Context(int(os.environ.get("LOCAL_RANK", 0)))
    try:
        r = mixbench.run_mix(ctx, args.scenes, args.steps, args.warmup)
    finally:
        ctx.close()
    torch.cuda.empty_cache()
    return {"unit": "scene-iters/s", "batched": r["value"], "plain_one_at_a_time": r["plain_seq_scene_iters_per_s"],
            "fused_one_at_a_time": r["fused_seq_scene_iters_per_s"], "ratio_vs_plain": r["speedup_vs_plain"],
            "ratio_vs_fused_one_at_a_time": r["speedup_vs_fused_seq"], "ms_per_batched_step": r["ms_per_step"],
            "steps": args.steps, "warmup": args.warmup, "launches_per_batched_step": r["launches_per_batched_step"],
            "one_at_a_time_by_resolution": r["one_at_a_time_by_resolution"], "subsets": r["subsets"],
            "first_step_ms_incl_autotune_capture": r["first_step_ms_incl_autotune_capture"],
            "workload": r["config"]["workload"], "resident_bytes": r["config"]["resident_bytes"]}


def serve_summary(args):
    """The serving loop at one arrival rate, repeated: median and range of
    p50/p99 job latency and iterations/s, beside the same jobs one at a time
    through the plain pipeline."""
    import torch
    from vcl_b200 import capi, mixbench
    ctx = capi.Context(int(os.environ.get("LOCAL_RANK", 0)))
    try:
        r = mixbench.run_serve(ctx, args.serve_jobs, [args.serve_lam], repeats=args.serve_repeats)
    finally:
        ctx.close()
    torch.cuda.empty_cache()
    sw = r["sweep"]

    def stat(key, src=None):
        xs = [(x[src] if src else x)[key] for x in sw]
        xs = [x for x in xs if x is not None]
        return {"median": statistics.median(xs), "min": min(xs), "max": max(xs)} if xs else None

    return {"lambda_per_s": args.serve_lam, "jobs": r["jobs"], "repeats": len(sw),
            "iterations_per_repeat": r["iterations_total"], "budget_gb": r["budget_gb"],
            "p50_ms": stat("p50_ms"), "p99_ms": stat("p99_ms"), "iters_per_s": stat("iters_per_s"),
            "completed": [x["completed"] for x in sw],
            "plain_one_at_a_time": {"p50_ms": stat("p50_ms", "plain_one_at_a_time"),
                                    "p99_ms": stat("p99_ms", "plain_one_at_a_time"),
                                    "iters_per_s": stat("iters_per_s", "plain_one_at_a_time")},
            "workload": f"{r['jobs']} fit jobs from the uneven scene mix, U[50,500] iterations each, Poisson "
                        f"arrivals at {args.serve_lam:g} jobs/s, {r['budget_gb']:g} GB admission budget"}


def config5_summary(args):
    """The dense-stress fit iteration (icosphere s8, 1,310,720 triangles, 4
    views of 2048^2, 4096^2 texture with 13 levels, 64 lobes), fused and
    plain, timed by this script in a child process (--config config5)."""
    cmd = [sys.executable, os.path.abspath(__file__), "--config", "config5", "--no-mix", "--no-serve",
           "--no-config5", "--no-cpu-baseline", "--no-e2e", "--steps", "10", "--warmup", "3"]
    out = subprocess.run(cmd, capture_output=True, text=True)
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    if out.returncode != 0 or not lines:
        raise RuntimeError(f"config5 run failed: {out.stderr[-2000:]}")
    d = json.loads(lines[-1])
    return {"workload": d["config"]["workload"], "iters_per_s": d["value"], "ms_per_step": d["ms_per_step"],
            "strategies_ms_per_step": d["strategies_ms_per_step"], "fused_kernels_ms": d.get("fused_kernels_ms"),
            "stages_ms": d.get("stages_ms"), "raster_ties": d.get("raster_ties"), "steps": 10, "warmup": 3,
            "clocks": d.get("clocks")}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ and args.impl != "reference":
        sys.exit(spawn_ranks(args.gpus))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args, rank, world)), flush=True)
        return
    if args.config in ("mix", "serve"):
        return run_mixed(args, rank, world)
    import torch
    from vcl_b200 import replicas
    if world > 1:
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        replicas.init("nccl", timeout_s=120)
    r = run_vcl(args, rank, world)
    replicas.finish()
    if rank != 0:
        return
    S = r["scene"]
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    line = {
        "metric": METRIC, "value": r["value"], "unit": "iters/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded; no dataset)",
        "config": bench_config(S, world),
        "strategy": r["best"],
        "strategies_ms_per_step": {k: v / args.steps for k, v in r["results"].items()},
        "gpu_launches": r["launches"][r["best"]] * args.steps,
        "clocks": r["clocks"],
        "e2e": None if r["e2e_ms"] is None else {
            "value": world * 1000.0 / r["e2e_ms"], "unit": "iters/s",
            "h2d_bytes_per_step": S.views * S.H * S.W * S.C * 4 + S.views * (16 + 9) * 4,
            "d2h_bytes_per_step": 4},
        # the end-to-end loop with the target images uploaded once: per step
        # only the cameras go host -> device and the loss comes back
        "e2e_targets_resident": None if r.get("e2e_resident_ms") is None else {
            "value": world * 1000.0 / r["e2e_resident_ms"], "unit": "iters/s",
            "h2d_bytes_per_step": S.views * (16 + 9) * 4, "d2h_bytes_per_step": 4},
        "loss_last": r["losses"][r["best"]],
        "raster_autotune": ({"tile": r["raster_tuning"][0],
                             "ms_per_tile_8_16_32": [round(x, 4) for x in r["raster_tuning"][1]]}
                            if "raster_tuning" in r else None),
    }
    ncov = r["stages"]["ncov"] if "stages" in r else S.W * S.H * S.views // 2
    if "fused_kernel_ms" in r:
        # the dominant kernel of the fused step, timed live (CUDA events on its
        # stream, after the timed region)
        kall = r["fused_kernel_ms"]
        byts = fused_bytes(S, ncov)
        kms = {k: v for k, v in kall.items() if k in byts}
        top = max(kms, key=lambda k: kms[k])
        b = byts[top]
        achieved = b / (kms[top] * 1e-3) / 1e9
        N = S.W * S.H * S.views
        traffic = DRAM_BYTES_PER_PIXEL[top] * N if top in DRAM_BYTES_PER_PIXEL else None
        line["roofline"] = {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                            "frac": achieved / hbm_peak, "traffic": traffic, "peak_source": peak_src,
                            "algorithmic_bytes": b, "avg_ms": kms[top],
                            "note": BOUND_NOTE.get(top)}
        line["fused_kernels_ms"] = {k: round(v, 4) for k, v in kall.items()}
        line["fused_kernels_frac_hbm"] = {k: round(byts[k] / (v * 1e-3) / 1e9 / hbm_peak, 3)
                                          for k, v in kms.items() if v > 0}
        # the SG kernels' own bound, the MUFU pipe: 2 rsqrt + 4 ex2 per covered
        # pixel and lobe in each, against the MUFU rate measured by the probe
        # on this GPU (the nominal 16 operations per clock per SM beside it)
        import torch
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        mhz = (r["clocks"] or {}).get("sm_mhz") or 1965.0
        nominal = 16.0 * sms * mhz * 1e6
        up = r.get("unit_peaks") or {}
        sfu_peak = up.get("mufu_ops_per_s") or nominal
        ops = 6.0 * ncov * S.K
        line["sfu_roofline"] = {
            k: {"mufu_ops": ops, "achieved_gops": ops / (kms[k] * 1e-3) / 1e9, "peak_gops": sfu_peak / 1e9,
                "frac": ops / (kms[k] * 1e-3) / sfu_peak, "covered_pixels": ncov,
                "peak_source": "measured (vcl_probe_mufu_throughput)" if "mufu_ops_per_s" in up else "nominal",
                "nominal_gops": nominal / 1e9}
            for k in ("shade_fwd", "sg_lobes") if kms.get(k, 0) > 0}
        # their other bound, the FP32 FMA pipe: FP32 operations per covered
        # pixel and lobe in the SG arithmetic as written (paired instructions
        # counted as two): 34 in the shading sums (two lobes per
        # instruction), 65 in the lobe gradients (COMPAT; two pixels per
        # instruction), against the paired-FMA rate measured by the probe
        fma_nominal = 128.0 * sms * mhz * 1e6
        fma_peak = up.get("fma_ops_per_s") or fma_nominal
        fma_ops = {"shade_fwd": 34.0 * ncov * S.K, "sg_lobes": 65.0 * ncov * S.K}
        line["fma_roofline"] = {
            k: {"fp32_ops": fma_ops[k], "achieved_gops": fma_ops[k] / (kms[k] * 1e-3) / 1e9,
                "peak_gops": fma_peak / 1e9, "frac": fma_ops[k] / (kms[k] * 1e-3) / fma_peak,
                "peak_source": "measured (vcl_probe_fma_throughput)" if "fma_ops_per_s" in up else "nominal",
                "nominal_gops": fma_nominal / 1e9}
            for k in ("shade_fwd", "sg_lobes") if kms.get(k, 0) > 0}
        if "l2_red_v4_per_s" in up and kms.get("bwd_pix", 0) > 0:
            # the per-pixel backward's texel scatter: 4 vector reductions per
            # covered pixel and level it samples (8 with trilinear sampling),
            # the reference's atomics per pixel (texturemap.cu:246-279), against
            # the measured L2 vector-reduction rate
            reds = 8.0 * ncov
            line["atomic_roofline"] = {
                "bwd_pix": {"texel_reductions": reds, "achieved_per_s": reds / (kms["bwd_pix"] * 1e-3),
                            "peak_per_s": up["l2_red_v4_per_s"],
                            "frac": reds / (kms["bwd_pix"] * 1e-3) / up["l2_red_v4_per_s"],
                            "peak_source": "measured (vcl_probe_red_throughput, coalesced)"}}
        line["unit_peaks"] = up
    if "stages" in r:
        st = r["stages"]
        byts = stage_bytes(S, st["ncov"])
        ms = st["ms"]
        if "roofline" not in line:
            top = max(ms, key=lambda k: ms[k])
            b = byts.get(top, 0)
            achieved = b / (ms[top] * 1e-3) / 1e9
            line["roofline"] = {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": hbm_peak,
                                "unit": "GB/s", "frac": achieved / hbm_peak, "traffic": None,
                                "peak_source": peak_src, "algorithmic_bytes": b, "avg_ms": ms[top]}
        line["stages_ms"] = {k: round(v, 4) for k, v in ms.items()}
        line["raster_ties"] = st.get("ties")
        line["stages_frac_hbm"] = {k: round(byts.get(k, 0) / (v * 1e-3) / 1e9 / hbm_peak, 3) for k, v in ms.items()
                                   if v > 0}
    if not args.no_cpu_baseline:
        # one full fit iteration of the workload (V view-steps) after one
        # warm-up step, on every host core
        per_iter, _, kind, cores, sample = time_reference(S, os.cpu_count() or 1, S.views, 1)
        line["cpu_baseline"] = {"value": 1.0 / per_iter, "unit": "iters/s", "cores": cores, "kind": kind,
                                "sample": sample}
    if not args.no_config5 and args.config == "config2":
        line["config5"] = config5_summary(args)
    if not args.no_mix:
        line["mix"] = mix_summary(args)
    if not args.no_serve:
        line["serve"] = serve_summary(args)
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
