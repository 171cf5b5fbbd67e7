"""Measurements of the batched engine and the serving loop on the uneven
scene mix (icospheres of 1k-200k triangles, 128^2-1024^2 x 1-16 views,
256^2-2048^2 textures, 8-32 lobes), called by ``bench.py --config mix`` and
``bench.py --config serve``.

mix    one batched launch per iteration of all scenes (vcl_batch_step)
       against the same scenes stepped one at a time, fused (each its own
       graph) and plain (one launch per operator).  Unit: scene
       fit-iterations per second.
serve  Poisson arrivals of fit jobs (rate swept), each job running
       U[50, 500] iterations on a scene of the mix, admitted by device
       footprint under a 150 GB budget and interleaved by vcl_server_tick;
       p50/p99 latency from arrival to completion and iterations per second.
       Beside it, the same jobs one at a time through the plain pipeline:
       every job is run to completion alone (set-up, all its iterations,
       loss read back) and timed, and the first-come-first-served timeline of
       one job at a time is computed from those durations and the same
       arrival times.
Targets are the true scene rendered on the device plus N(0, 0.05) noise.
"""
import time

import numpy as np


def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def render_targets(ctx, capi, torch, scenes_, stream, host=False, noise=0.05):
    """True-scene renders + noise, on the device (or copied to host)."""
    out = []
    sh = stream.cuda_stream
    for i, S in enumerate(scenes_):
        truth = capi.Fit(ctx, S, tex=S.tex_target, pos=S.pos_target,
                         lobes=(S.lobe_axis, S.lobe_sharp, S.lobe_amp), learn=(0, 0, 0))
        n = S.W * S.H * S.views * S.C
        t = torch.empty(n, dtype=torch.float32, device="cuda")
        with torch.cuda.stream(stream):
            truth.render(t, sh)
            g = torch.Generator(device="cuda").manual_seed(1000 + i)
            t.add_(torch.randn(n, generator=g, device="cuda") * noise)
        stream.synchronize()
        truth.close()
        out.append(t.cpu().numpy() if host else t)
    return out


def run_mix(ctx, n_scenes, steps, warmup, seed=0):
    import torch
    from vcl_b200 import capi, scenes
    S_list = scenes.config3(seed=seed, n=n_scenes)
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    targets = render_targets(ctx, capi, torch, S_list, stream)
    fits = []
    for S, t in zip(S_list, targets):
        f = capi.Fit(ctx, S, strategy=capi.FIT_FUSED)
        f.set_target(t, sh, is_device=True)
        fits.append(f)
    stream.synchronize()
    batch = capi.Batch(ctx)
    for f in fits:
        batch.add(f)
    t0 = time.perf_counter()
    batch.step(sh)              # autotune + capture + instantiate happen here
    stream.synchronize()
    first_ms = (time.perf_counter() - t0) * 1e3
    for _ in range(max(0, warmup - 1)):
        batch.step(sh)
    stream.synchronize()
    e0, e1 = _events(torch)
    e0.record(stream)
    for _ in range(steps):
        batch.step(sh)
    e1.record(stream)
    stream.synchronize()
    batched_ms = e0.elapsed_time(e1) / steps
    launches = batch.launches_per_step()

    def seq(strategy, reps=2):
        tot = 0.0
        per = []
        for f in fits:
            f.set_strategy(strategy)
            f.step(sh)
            stream.synchronize()
            a, b = _events(torch)
            a.record(stream)
            for _ in range(reps):
                f.step(sh)
            b.record(stream)
            stream.synchronize()
            ms = a.elapsed_time(b) / reps
            per.append(ms)
            tot += ms
        return tot, per

    for f in fits:
        batch.remove(f)
    batch.close()

    # the same batched launch on the small scenes alone and on the large ones
    # alone: where batching pays (many small launches) and where it cannot
    # (kernels that already fill the GPU)
    def batched_subset(sel):
        sub = [f for f, S in zip(fits, S_list) if sel(S)]
        if not sub:
            return None, 0
        b = capi.Batch(ctx)
        for f in sub:
            b.add(f)
        for _ in range(max(1, warmup)):
            b.step(sh)
        stream.synchronize()
        a, z = _events(torch)
        a.record(stream)
        for _ in range(steps):
            b.step(sh)
        z.record(stream)
        stream.synchronize()
        for f in sub:
            b.remove(f)
        b.close()
        return a.elapsed_time(z) / steps, len(sub)

    small = lambda S: S.W * S.H <= 256 * 256
    subsets = {}
    for name, sel in (("small_256_or_less", small), ("large_512_or_more", lambda S: not small(S))):
        ms, n_sub = batched_subset(sel)
        subsets[name] = {"scenes": n_sub, "batched_ms": ms}
    fused_seq_ms, fused_per = seq(capi.FIT_FUSED)
    plain_seq_ms, plain_per = seq(capi.FIT_PLAIN)
    # where the time goes: scenes grouped by resolution, one at a time
    buckets = {}
    for S, pm, fm in zip(S_list, plain_per, fused_per):
        b = buckets.setdefault(f"{S.W}x{S.H}", {"scenes": 0, "pixels": 0, "triangles": 0, "plain_ms": 0.0,
                                                 "fused_ms": 0.0})
        b["scenes"] += 1
        b["pixels"] += S.W * S.H * S.views
        b["triangles"] += S.nt
        b["plain_ms"] += pm
        b["fused_ms"] += fm
    for b in buckets.values():
        b["plain_ms"] = round(b["plain_ms"], 3)
        b["fused_ms"] = round(b["fused_ms"], 3)
    for name, sel in (("small_256_or_less", small), ("large_512_or_more", lambda S: not small(S))):
        d = subsets[name]
        d["plain_one_at_a_time_ms"] = sum(pm for S, pm in zip(S_list, plain_per) if sel(S))
        d["fused_one_at_a_time_ms"] = sum(fm for S, fm in zip(S_list, fused_per) if sel(S))
        d["pixels"] = sum(S.W * S.H * S.views for S in S_list if sel(S))
        if d["batched_ms"]:
            d["ratio_vs_plain"] = d["plain_one_at_a_time_ms"] / d["batched_ms"]
    sched = {}
    for f in fits:
        f.set_strategy(capi.FIT_FUSED)
        t, sa, cap, cached, _ = f.raster_schedule()
        sched[f"{t}/{sa}"] = sched.get(f"{t}/{sa}", 0) + 1
    px = sum(S.W * S.H * S.views for S in S_list)
    resident = sum(capi.footprint(S) for S in S_list)
    for f in fits:
        f.close()
    n = len(S_list)
    return {
        "value": n * 1000.0 / batched_ms, "unit": "scene-iters/s", "ms_per_step": batched_ms,
        "plain_seq_scene_iters_per_s": n * 1000.0 / plain_seq_ms,
        "fused_seq_scene_iters_per_s": n * 1000.0 / fused_seq_ms,
        "speedup_vs_plain": plain_seq_ms / batched_ms, "speedup_vs_fused_seq": fused_seq_ms / batched_ms,
        "gpu_launches": launches * steps, "launches_per_batched_step": launches,
        "first_step_ms_incl_autotune_capture": round(first_ms, 1),
        "raster_schedules_tile_direct_area": sched,
        "subsets": subsets,
        "one_at_a_time_by_resolution": dict(sorted(buckets.items(), key=lambda kv: int(kv[0].split("x")[0]))),
        "config": {"workload": f"{n} uneven scenes (icosphere 1k-200k tris, 128^2-1024^2 x 1-16 views, "
                               f"256^2-2048^2 RGBA textures, 8-32 lobes), {px / 1e6:.1f} M pixels per iteration",
                   "scenes": n, "pixels": px, "resident_bytes": resident, "seed": seed},
    }


def run_serve(ctx, n_jobs, lams, budget_gb=150.0, seed=0, max_live=64, iters_range=(50, 500), repeats=1):
    import torch
    from vcl_b200 import capi, scenes
    rng = np.random.default_rng(seed + 7)
    S_list = [scenes.config3_scene(seed + 100, i) for i in range(n_jobs)]
    iters = [int(x) for x in rng.integers(iters_range[0], iters_range[1] + 1, size=n_jobs)]
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    targets = render_targets(ctx, capi, torch, S_list, stream, host=True)
    # plain, one job at a time: every job run to completion (set-up, all its
    # iterations, the loss read back), timed on the host clock
    plain_job_ms = []
    for S, t, n_it in zip(S_list, targets, iters):
        t0 = time.perf_counter()
        f = capi.Fit(ctx, S, strategy=capi.FIT_PLAIN)
        f.set_target(t)
        for _ in range(n_it):
            f.step(sh)
        f.read_loss(sh)
        plain_job_ms.append((time.perf_counter() - t0) * 1e3)
        f.close()
    out = {"jobs": n_jobs, "iterations_total": int(sum(iters)), "budget_gb": budget_gb, "max_live": max_live,
           "sweep": []}
    for lam in [l for l in lams for _ in range(repeats)]:
        arr = np.cumsum(rng.exponential(1000.0 / lam, size=n_jobs))   # ms after start
        srv = capi.Server(ctx, int(budget_gb * 1e9), max_live=max_live)
        base = srv.now_ms()
        ids = [None] * n_jobs
        nxt = 0
        t_start = time.perf_counter()
        while True:
            now = srv.now_ms() - base
            while nxt < n_jobs and arr[nxt] <= now:
                ids[nxt] = srv.submit(S_list[nxt], targets[nxt], iters[nxt])
                nxt += 1
            if nxt < n_jobs and srv.pending() == 0:
                time.sleep(max(0.0, (arr[nxt] - now) / 1000.0))
                continue
            srv.tick(sh)
            if nxt == n_jobs and srv.pending() == 0:
                break
        wall = time.perf_counter() - t_start
        lat = []
        for i, jid in enumerate(ids):
            s = srv.status(jid)
            if s["state"] == capi.JOB_DONE:
                lat.append(s["done_ms"] - (base + arr[i]))
        st = srv.stats()
        hs = srv.host_stats()
        srv.close()
        # plain one at a time, first come first served
        end, plat = 0.0, []
        for i in range(n_jobs):
            start = max(arr[i], end)
            end = start + plain_job_ms[i]
            plat.append(end - arr[i])
        span_plain = end - arr[0]
        lat = np.array(lat)
        out["sweep"].append({
            "lambda_per_s": lam, "completed": int(len(lat)),
            "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
            "iters_per_s": st["iterations"] / wall, "ticks": st["ticks"], "wall_s": wall,
            "host": {k: round(v, 1) for k, v in hs.items()},
            "plain_one_at_a_time": {"p50_ms": float(np.percentile(plat, 50)), "p99_ms": float(np.percentile(plat, 99)),
                                    "iters_per_s": sum(iters) / (span_plain / 1000.0)},
        })
    return out
