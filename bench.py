"""Benchmark of the gs_b200 frame pipeline on the headline workload:
3M Gaussians, SH degree 3, 64 views on an orbit ring at 1280x720 /
1600x900 / 1920x1080, all rendered as one batched frame.  A step is one
batched frame of the 64 views; the metric is views/s (whole job).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU (torchrun for N > 1).  Views shard across ranks as
independent replicas (each rank renders its own 64-view batch of the
resident scene; there is no collective in the frame), so scaling is weak.
--impl reference times the CPU rendition of the same pipeline (the oracle
restatement of the reference's stages, OpenMP over the host cores) on a
bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import datetime
import importlib
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

VIEWS = 64
N_GAUSS = 3_000_000
# DRAM bytes (read + written) of the T_min raster launch of view 0 (1280x720)
# rendered alone: ncu capture of the second frame of `bench.py --views 1
# --steps 1 --warmup 1 --no-cpu --no-e2e --no-plain --no-serve` (128.2 MB
# read, 7.0 MB written; the raster roofline's traffic)
RASTER_VIEW0_TRAFFIC = 133.7e6
RING_RADIUS = 15.0
WORKLOAD = "3M Gaussians SH3, 64-view orbit ring r=15, 1280x720/1600x900/1920x1080 cycling, one batched frame"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def make_workload(gs, rank=0):
    sc = gs.scenes.config_scene("batch3m")
    eyes = gs.scenes.orbit_ring(VIEWS, RING_RADIUS, seed=1000 + rank)
    cams = []
    for i, e in enumerate(eyes):
        W, H = gs.scenes.BATCH_RESOLUTIONS[i % 3]
        cams.append(gs.look_at(e, (0, 0, 0), (0, 1, 0), 50.0, W, H, 0.1, 100.0))
    return sc, cams


def scenes_module():
    """The seeded scene generator (plain numpy), loaded from its file so that
    the reference arm never loads the product library."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("gs_scenes", os.path.join(ROOT, "3dgaussianrenderer_b200",
                                                                            "scenes.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def make_workload_reference(O, rank=0):
    """make_workload's scene and cameras built without the product library:
    the same generator, cameras from the oracle's look-at (bit-identical to
    gs_camera_look_at, tests/test_oracle_cpu.py)."""
    sc_mod = scenes_module()
    sc = sc_mod.config_scene("batch3m")
    eyes = sc_mod.orbit_ring(VIEWS, RING_RADIUS, seed=1000 + rank)
    cams = [O.look_at(e, (0, 0, 0), (0, 1, 0), 50.0, *sc_mod.BATCH_RESOLUTIONS[i % 3], 0.1, 100.0)
            for i, e in enumerate(eyes)]
    return sc_mod, sc, cams


class Clocks:
    """nvidia-smi sampling (100 ms period) kept to the samples taken inside
    the timed region [mark_start(), mark_end()]."""

    def __init__(self, index=0):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        self.t0 = self.t1 = None
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(1.0)  # the sampler's own start-up
        except FileNotFoundError:
            self.p = None

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        self.f.seek(0)
        rows = [[x.strip() for x in r.split(",")] for r in self.f.read().strip().splitlines() if r.count(",") >= 9]
        os.unlink(self.f.name)

        def stamp(r):
            try:
                return datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except ValueError:
                return None

        if self.t0 is not None and self.t1 is not None:
            inside = [r for r in rows if stamp(r) is not None and self.t0 - 0.05 <= stamp(r) <= self.t1 + 0.05]
            if inside:
                rows = inside
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        mx = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, nm in enumerate(names):
                if "Active" in r[6 + k] and "Not" not in r[6 + k]:
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def cpu_baseline(gs, sc, cams, rc, sample_views=1, threads=None):
    """The oracle (CPU rendition of the five stages) over a bounded sample of
    views, with the render options of the GPU leg."""
    import oracle
    O = oracle.get()
    if threads:
        O.set_threads(threads)
    sh = gs.scenes.grouped_sh(sc["sh"])
    t0 = time.perf_counter()
    for v in range(sample_views):
        O.render(sc, sh, cams[v], rc)
    dt = time.perf_counter() - t0
    # work of view 0 for the raster roofline (outside the timed sample):
    # evaluations of every splat until T < t_min, and those the GPU's
    # warp-culled raster executes
    O.count_block_evals(True)
    _, _, evals, _ = O.render(sc, sh, cams[0], rc)
    block_evals = O.block_evals()
    O.count_block_evals(False)
    return {"value": sample_views / dt, "unit": "views/s", "cores": O.max_threads(), "kind": "port",
            "sample": f"{sample_views} of the 64 views ({cams[0].GetWidth()}x{cams[0].GetHeight()}), full frame "
                      f"(SH3 + project + build + sort + raster) of the 3M scene, {dt:.1f} s",
            "evals_view0": evals, "block_evals_view0": block_evals}


SERVE_SCENES = [200_000, 500_000, 1_000_000, 1_000_000, 2_000_000, 2_000_000, 3_000_000, 4_000_000]
SERVE_RES = [(1280, 720), (1920, 1080), (2560, 1440)]


def run_serving(gs, rank, rates=(500.0, 2000.0, 5000.0), requests=10_000, budget_gb=150, max_batch=16, workers=2):
    """Serving workload: 8 resident scenes, Poisson request streams at each
    of `rates` req/s in turn (scene uniform, pose uniform on a radius-12
    sphere, resolution uniform over 720p/1080p/1440p), admitted against a
    device-memory budget; `requests` requests per rate (about 20 s at 500
    req/s, the configuration's rate; the faster streams show continuous
    batching under load).  Latency = submit -> image in host memory."""
    srv = gs.Server(0, budget_bytes=budget_gb << 30, max_batch_views=max_batch, num_workers=workers)
    ids = []
    for k, n in enumerate(SERVE_SCENES):
        sc = gs.scenes.cluster_scene(n, 256, 10.0, seed=500 + 17 * rank + k)
        ids.append(srv.add_scene(sc["pos4"], sc["sr4"], gs.scenes.grouped_sh(sc["sh"]), 3))
        del sc
    import torch
    rng = np.random.default_rng(77 + rank)
    ring = 64
    # pinned host buffers: the images are copied straight into them
    bufs = [torch.empty(2560 * 1440 * 4, dtype=torch.uint8).pin_memory().numpy() for _ in range(ring)]
    inflight = [None] * ring

    def make_request():
        s = ids[int(rng.integers(0, len(ids)))]
        W, H = SERVE_RES[int(rng.integers(0, len(SERVE_RES)))]
        cam = gs.look_at(gs.scenes.sphere_pose(rng, 12.0), (0, 0, 0), (0, 1, 0), 50.0, W, H, 0.1, 100.0)
        return s, cam

    # warm-up: every scene and resolution once, then full-size bursts of the
    # largest scene so every worker's frame buffers reach their steady size
    for s in ids:
        for (W, H) in SERVE_RES:
            cam = gs.look_at((0.0, 1.0, 12.0), (0, 0, 0), (0, 1, 0), 50.0, W, H, 0.1, 100.0)
            srv.wait(srv.submit(s, cam, bufs[0]))
    for _ in range(3):
        burst = []
        for k in range(min(ring, workers * max_batch)):
            cam = gs.look_at(gs.scenes.sphere_pose(rng, 12.0), (0, 0, 0), (0, 1, 0), 50.0, 2560, 1440, 0.1, 100.0)
            burst.append(srv.submit(ids[-1], cam, bufs[k]))
        for r in burst:
            srv.wait(r)
    legs = []
    for rate in rates:
        srv.reset_stats()
        t0 = time.perf_counter()
        t_next = t0
        slot = 0
        count = 0
        while count < requests:
            t_next += rng.exponential(1.0 / rate)
            s, cam = make_request()
            if inflight[slot] is not None:
                srv.wait(inflight[slot])
                inflight[slot] = None
            delay = t_next - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            inflight[slot] = srv.submit(s, cam, bufs[slot])
            slot = (slot + 1) % ring
            count += 1
        for k, r in enumerate(inflight):
            if r is not None:
                srv.wait(r)
                inflight[k] = None
        st = srv.stats()
        legs.append({"views_per_s": st["views_per_s"], "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
                     "mean_ms": st["mean_ms"], "requests": count, "rate_req_s": rate, "max_batch": st["max_batch"],
                     "batches": st["batches_done"]})
    srv.close()
    out = dict(legs[0], budget_gb=budget_gb, workers=workers, in_flight_limit=ring,
               scenes_m=[n / 1e6 for n in SERVE_SCENES])
    out["sweep"] = legs[1:]
    return out


def job_views_per_s(local_ms: float, views_per_rank: int, steps: int, world: int, device=None) -> tuple:
    """Whole-job throughput of `world` replicas: every rank renders its own
    views (no exchange), the job takes as long as the slowest rank, so
    value = all ranks' views / max over ranks of the timed milliseconds.
    Returns (value, max_ms); a collective only when world > 1."""
    import torch
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    return world * views_per_rank * steps / (ms_max / 1e3), ms_max


def run_ref1024(gs, ctx, sc, dev, stream, frames=30):
    """The single-view path in reference-compatible mode (SH degree <= 2 as
    the reference evaluates it, tile-wide T <= 0.02 termination) on the same
    3M-Gaussian scene at 1024x1024, the only size the reference renders:
    the frame the reference's own CUDA pipeline is compared with.  Median of
    `frames` frames, CUDA events around each frame call."""
    import torch
    eye = gs.scenes.orbit_ring(64, RING_RADIUS, seed=1000)[0]
    cam = gs.look_at(eye, (0, 0, 0), (0, 1, 0), 50.0, 1024, 1024, 0.1, 100.0)
    sh = gs.scenes.grouped_sh(sc["sh"])
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], sh, 3)
    rc = gs.RenderConfig.reference()
    out = torch.empty((1024, 1024, 4), dtype=torch.uint8, device=dev)
    for _ in range(3):
        gs.render(ctx, scene, cam, rc, out, stream)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(frames)]
    st = None
    for a, b in ev:
        a.record(stream)
        st = gs.render(ctx, scene, cam, rc, out, stream)
        b.record(stream)
    torch.cuda.synchronize()
    ms = float(np.median([a.elapsed_time(b) for a, b in ev]))
    scene.close()
    return {"frame_ms": ms, "keys": st["num_keys"], "workload": "3M Gaussians SH3 (clusters), 1024x1024, "
            "reference-compatible mode, single view"}


def run_ref_cuda_1024(sc, frames=30):
    """The reference's own CUDA frame (its kernels built from
    core/gaussian_render.cu into oracle/_ref/libgsref.so, run by the headless
    frame loop of app/main.cpp:360-432) on the same 3M-Gaussian scene and
    1024x1024 camera as run_ref1024, on the same GPU, in the same process:
    the comparison the plain path's >= 1.5x target is quoted against.  Median
    of `frames` frames, CUDA events around each whole frame.  None when the
    harness was not built (the reference sources were absent)."""
    import oracle
    if not os.path.exists(oracle.REF_LIB):
        return None
    O = oracle.get()
    sc_mod = scenes_module()
    eye = sc_mod.orbit_ring(64, RING_RADIUS, seed=1000)[0]
    cam = O.look_at(eye, (0, 0, 0), (0, 1, 0), 50.0, 1024, 1024, 0.1, 100.0)
    ref = oracle.Ref()
    _, k, times, stage = ref.time_frames(sc["pos4"], sc["sr4"], sc_mod.grouped_sh(sc["sh"]), 3, cam, frames)
    return {"frame_ms": float(np.median(times)), "keys": k,
            "stage_ms_sh_clip_build_sort_ranges_raster": stage,
            "workload": "the reference's CUDA frame loop (SH degree <= 2, tile-wide T <= 0.02), same scene and "
                        "camera"}


def run_sort_vs_cub(gs, ctx, sc, dev, iters=15):
    """The onesweep sort of gs_stage_sort against the sort the reference
    calls, CUB's DeviceRadixSort::SortPairs (its sortTileList,
    core/gaussian_render.cu:591-632, built into oracle/_ref/libgsref.so), on
    identical (key, value) pairs and key widths, each call timed with CUDA
    events after the unsorted input is restored: the tile-list keys of the
    1024x1024 reference-mode frame of the 3M scene (44 bits, the reference's
    width) and 222M random keys of the 64-view batch's width (51 bits).  The
    outputs must be identical (both sorts are stable).  Median ms per sort."""
    import ctypes
    import torch
    import oracle
    if not os.path.exists(oracle.REF_LIB):
        return None
    ref = oracle.Ref()
    out = []
    # keys of the 1024^2 frame: the stage API's projection and build
    eye = gs.scenes.orbit_ring(64, RING_RADIUS, seed=1000)[0]
    cam = gs.look_at(eye, (0, 0, 0), (0, 1, 0), 50.0, 1024, 1024, 0.1, 100.0)
    n = sc["pos4"].shape[0]
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    xy = torch.zeros((n, 2), dtype=torch.float32, device=dev)
    z = torch.zeros(n, dtype=torch.float32, device=dev)
    ell = torch.zeros((n, 4), dtype=torch.float32, device=dev)
    con = torch.zeros((n, 4), dtype=torch.float32, device=dev)
    gs.stage_project(n, t(sc["pos4"]), t(sc["sr4"]), cam, xy, z, ell, con)
    cap = 16 * n
    k = torch.zeros(cap, dtype=torch.int64, device=dev)
    v = torch.zeros(cap, dtype=torch.int32, device=dev)
    K = gs.stage_build(ctx, n, xy, z, ell, cam, gs.RenderConfig.reference(), k, v, cap)
    del xy, z, ell, con
    cases = [("1024x1024 frame keys, 3M scene", k[:K].clone(), v[:K].clone(), 44)]
    del k, v
    m = 222_000_000
    g = torch.Generator(device=dev)
    g.manual_seed(5)
    rk = (torch.randint(0, 1 << 19, (m,), device=dev, generator=g, dtype=torch.int64) << 32) | \
        torch.randint(0, 1 << 32, (m,), device=dev, generator=g, dtype=torch.int64)
    rv = torch.arange(m, dtype=torch.int32, device=dev)
    cases.append(("222M random keys (64-view batch width)", rk, rv, 51))
    for name, src_k, src_v, bits in cases:
        cnt = src_k.numel()
        k0, k1 = torch.empty_like(src_k), torch.empty_like(src_k)
        v0, v1 = torch.empty_like(src_v), torch.empty_like(src_v)
        sel = ctypes.c_int(0)
        cub_ms = ref.lib.gsref_cub_sort_timed(cnt, bits, src_k.data_ptr(), src_v.data_ptr(), k0.data_ptr(),
                                              k1.data_ptr(), v0.data_ptr(), v1.data_ptr(), iters, ctypes.byref(sel))
        torch.cuda.synchronize()
        cub_k = (k1 if sel.value else k0).clone()
        cub_v = (v1 if sel.value else v0).clone()
        # the same restore-then-time protocol, around the sort alone
        s_ours, ours_ms = gs.probe_sort_timed(ctx, cnt, bits, src_k, src_v, k0, v0, k1, v1, iters)
        torch.cuda.synchronize()
        ours_k = k1 if s_ours else k0
        ours_v = v1 if s_ours else v0
        same = bool(torch.equal(ours_k, cub_k) and torch.equal(ours_v, cub_v))
        out.append({"case": name, "keys": int(cnt), "bits": bits, "cub_ms": float(cub_ms), "ours_ms": ours_ms,
                    "speedup": float(cub_ms) / ours_ms, "identical_output": same,
                    "ours_gkeys_s": cnt / ours_ms / 1e6})
        del k0, k1, v0, v1, cub_k, cub_v
    return out


def run_reference(args, rank, world):
    if rank != 0:
        return
    import oracle
    O = oracle.get()
    sc_mod, sc, cams = make_workload_reference(O)
    sh = sc_mod.grouped_sh(sc["sh"])
    # the frame options of the GPU leg: SH degree 3, per-pixel T < 1e-4, 16x16 tiles
    rc = oracle.gso_cfg(3, 1, 1e-4, 16, 16)
    for w in range(args.warmup):
        O.render(sc, sh, cams[w % VIEWS], rc)
    times = []
    for s in range(args.steps):
        t0 = time.perf_counter()
        O.render(sc, sh, cams[s % VIEWS], rc)
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    value = args.steps / tot
    line = {
        "impl": "reference", "metric": "views/s", "value": value, "unit": "views/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "step": "one view of the workload rendered on the host cores",
                   "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": value, "unit": "views/s", "cores": O.max_threads(), "kind": "port",
                         "sample": "each step renders one of the 64 views (full frame, SH3) with the oracle "
                                   "restatement of the reference stages, OpenMP"},
        "e2e": {"value": value, "unit": "views/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    gs = importlib.import_module("3dgaussianrenderer_b200")
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    ctx = gs.Context(local_rank)
    sc, cams = make_workload(gs, rank)
    stream = torch.cuda.current_stream(dev)
    if args.only_ref1024:
        # profiling case: the reference-compatible 1024x1024 frame alone
        r = run_ref1024(gs, ctx, sc, dev, stream, frames=args.steps)
        if rank == 0:
            print(json.dumps({"metric": "frame_ms", "value": r["frame_ms"], "unit": "ms", "higher_is_better": False,
                              "config": r}), flush=True)
        ctx.close()
        return
    sh = gs.scenes.grouped_sh(sc["sh"])
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], sh, 3)
    rc = gs.RenderConfig()
    tuned = None
    if not args.no_autotune:
        # the project's autotuner picks the knobs (tile shape, views per
        # block, ordering, the tile sort's radix width, the raster's batch of
        # Gaussians, the persistent raster) for this (N, resolution, views)
        # bucket by coordinate descent, outside the timed region; every rank
        # tunes its own replica
        best, best_ms, cands = gs.autotune(ctx, scene, cams, gs.RenderConfig(ordering=gs.GS_ORDER_AUTO),
                                           iterations=3, stream=stream)
        rc = best

        def knobs(c):
            return {"tile": f"{c.tile_w}x{c.tile_h}", "views_per_block": c.views_per_block,
                    "ordering": "onesweep" if c.ordering == gs.GS_ORDER_ONESWEEP else "buckets",
                    "sort_variant": c.sort_variant, "sort_bits": c.sort_bits, "raster_chunk": c.raster_chunk,
                    "raster_persistent": c.raster_persistent}

        tuned = {"picked": dict(knobs(best), ms=best_ms), "search": "coordinate descent",
                 "candidates": [dict(knobs(c), ms=m) for c, m in cands]}
    outs = [torch.empty((c.GetHeight(), c.GetWidth(), 4), dtype=torch.uint8, device=dev) for c in cams]

    def step():
        return gs.render_batch(ctx, scene, cams, rc, outs, stream)

    for _ in range(args.warmup):
        st = step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = Clocks(local_rank) if rank == 0 else None
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    stages = {"project_ms": 0.0, "build_tile_ms": 0.0, "sort_ms": 0.0, "raster_ms": 0.0}
    launches = 0
    keys = 0
    if clk:
        clk.mark_start()
    e0.record(stream)
    for _ in range(args.steps):
        st = step()
        for k in stages:
            stages[k] += st[k]
        launches += st["kernel_launches"]
        keys = st["num_keys"]
    e1.record(stream)
    torch.cuda.synchronize()
    if clk:
        clk.mark_end()
    ms = e0.elapsed_time(e1)
    clocks = clk.stop() if clk else None
    value, ms_max = job_views_per_s(ms, VIEWS, args.steps, world, dev)

    # e2e through the public host-buffer API: camera upload + images back to pinned host memory
    total_bytes = sum(c.GetWidth() * c.GetHeight() * 4 for c in cams)
    e2e_value = None
    if not args.no_e2e:
        host = torch.empty(total_bytes, dtype=torch.uint8).pin_memory()
        host_np = host.numpy()
        # a frame is captured into a CUDA graph on its second call: warm up
        # past that, as for the device-output leg
        for _ in range(max(3, args.warmup)):
            gs.render_batch_host(ctx, scene, cams, rc, host_np, stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            gs.render_batch_host(ctx, scene, cams, rc, host_np, stream)
        f1.record(stream)
        torch.cuda.synchronize()
        e2e_value, _ = job_views_per_s(f0.elapsed_time(f1), VIEWS, args.steps, world, dev)

    # plain single-view path over the same views (for the batched/plain ratio)
    plain_value = None
    raster_view0_ms = None
    if not args.no_plain:
        plain_views = min(VIEWS, 16)
        for v in range(2):
            gs.render(ctx, scene, cams[v], rc, outs[v], stream)
        torch.cuda.synchronize()
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for v in range(plain_views):
            gs.render(ctx, scene, cams[v], rc, outs[v], stream)
        g1.record(stream)
        torch.cuda.synchronize()
        plain_value = plain_views / (g0.elapsed_time(g1) / 1e3)
        # raster stage of view 0 alone (the raster roofline below)
        r0 = []
        for _ in range(10):
            r0.append(gs.render(ctx, scene, cams[0], rc, outs[0], stream)["raster_ms"])
        raster_view0_ms = float(np.median(r0))

    ref1024 = None
    if not args.no_plain:
        clk1024 = Clocks(local_rank) if rank == 0 else None
        if clk1024:
            clk1024.mark_start()
        ref1024 = run_ref1024(gs, ctx, sc, dev, stream)
        if rank == 0 and not args.no_ref_cuda:
            # the reference's own CUDA frame on the same scene, camera and GPU
            rc_ref = run_ref_cuda_1024(sc)
            if rc_ref:
                ref1024["ref_cuda_1024_frame_ms"] = rc_ref["frame_ms"]
                ref1024["ref_cuda_1024"] = rc_ref
                ref1024["speedup_vs_ref_cuda"] = rc_ref["frame_ms"] / ref1024["frame_ms"]
                ref1024["same_keys_as_ref_cuda"] = rc_ref["keys"] == ref1024["keys"]
        if clk1024:
            clk1024.mark_end()
            ref1024["clocks"] = clk1024.stop()

    sort_vs_cub = None
    if rank == 0 and not args.no_ref_cuda and not args.no_plain:
        clk_sort = Clocks(local_rank)
        clk_sort.mark_start()
        sort_vs_cub = run_sort_vs_cub(gs, ctx, sc, dev)
        clk_sort.mark_end()
        clocks_sort = clk_sort.stop()
        if sort_vs_cub:
            sort_vs_cub = {"cases": sort_vs_cub, "clocks": clocks_sort}
        torch.cuda.empty_cache()

    served = None
    if not args.no_serve:
        # release this leg's frame buffers first: the server has its own
        del outs
        ctx.close()
        scene.close()
        torch.cuda.empty_cache()
        served = run_serving(gs, rank)

    if rank != 0:
        return
    hbm, peak_kind = peaks()
    per = {k: v / args.steps for k, v in stages.items()}
    K = keys
    # Frame kernel against HBM.  Algorithmic bytes of one launch: the scene
    # (32 B position + scale/rotation, 12 (d + 1)^2 = 192 B SH per Gaussian)
    # read once per block of `vpb` views, and the 48-byte splat record per
    # (view, Gaussian) of the scope table written: ceil(V / vpb) N 224 + V N 48.
    # traffic: DRAM bytes of an ncu capture of a 4-view frame (684.2 MB read,
    # 506.1 MB written), scaled to 64 views (reads per block of views, writes
    # per view).  The kernel is issue-bound, far under this roof.
    vpb = min(VIEWS, rc.views_per_block or 16)
    blocks = (VIEWS + vpb - 1) // vpb
    alg_frame = blocks * N_GAUSS * (32 + 12 * 16) + VIEWS * N_GAUSS * 48
    frame_traffic = 684.2e6 * blocks + 506.1e6 / 4 * VIEWS if VIEWS == 64 else None
    frame_gbs = alg_frame / (per["project_ms"] / 1e3) / 1e9 if per["project_ms"] > 0 else None
    frame_roof = {"bound": "hbm", "kernel": "frame_project (SH + projection + tile counts)",
                  "achieved": frame_gbs, "peak": hbm, "unit": "GB/s",
                  "frac": frame_gbs / hbm if frame_gbs else None, "traffic": frame_traffic,
                  "algorithmic_bytes": alg_frame,
                  "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind}
    dom = max(per, key=per.get)
    cpu = cpu_baseline(gs, sc, cams, rc, sample_views=1) if (world == 1 and not args.no_cpu) else None
    # The dominant kernel, the T_min raster, against the FP32 pipe (it is
    # neither HBM- nor tensor-bound), for view 0 rendered alone, with the
    # scope table's fixed count: 20 FP32 flop per (pixel, splat) blend
    # evaluation (the reference's expression: offset, quadratic form,
    # exponent scale, alpha, three colour multiply-adds and the
    # transmittance update, a multiply-add counted as 2), over the
    # evaluations the GPU's warp-culled walk executes as counted by the
    # oracle's model of it; time = the raster stage; peak = 148 SMs x 128
    # FP32 lanes x 2 flop x the SM clock sampled during the timed region
    # (nominal: there is no measured FP32 peak).  The oracle's count without
    # the cull (every entry until T < t_min) is given beside it.  traffic:
    # DRAM bytes of an ncu capture of the same single-view launch.
    raster_roof = None
    if cpu and cpu.get("block_evals_view0") and raster_view0_ms:
        clk_mhz = (clocks or {}).get("sm_mhz") or 1965.0
        peak_gflops = 148 * 128 * 2 * clk_mhz * 1e6 / 1e9
        ach = 20.0 * cpu["block_evals_view0"] / (raster_view0_ms / 1e3) / 1e9
        raster_roof = {"bound": "fp32", "kernel": "raster_rec (T_min records, per-tile sort fused)",
                       "achieved": ach, "peak": peak_gflops, "unit": "GFLOP/s", "frac": ach / peak_gflops,
                       # captured with 16x16 tiles
                       "traffic": RASTER_VIEW0_TRAFFIC if (rc.tile_w, rc.tile_h) == (16, 16) else None,
                       "evals_executed": cpu["block_evals_view0"], "evals_unculled": cpu["evals_view0"],
                       "flop_per_eval": 20, "raster_ms": raster_view0_ms,
                       "view": f"view 0 ({cams[0].GetWidth()}x{cams[0].GetHeight()}) rendered alone",
                       "peak_kind": "nominal: 148 SMs x 128 FP32 lanes x 2 flop x sampled SM clock"}
    roof = raster_roof or frame_roof
    roof = dict(roof, stage_ms=per, dominant_stage=dom)
    line = {
        "metric": "views/s", "value": value, "unit": "views/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "views_per_step": VIEWS, "gaussians": N_GAUSS, "sh_degree": 3,
                   "termination": "per-pixel T<1e-4", "tiles": f"{rc.tile_w}x{rc.tile_h}",
                   "views_per_block": rc.views_per_block or 16, "autotune": tuned, "keys_per_step": K,
                   "l2": "inputs larger than L2 (scene 672 MB, per-view buffers ~15 GB)", "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e_value, "unit": "views/s", "h2d_bytes_per_step": VIEWS * 200,
                "d2h_bytes_per_step": total_bytes},
        "plain_views_per_s": plain_value,
        "batched_over_plain": (value / world / plain_value) if plain_value else None,
        "plain_ref_mode_1024": ref1024,
        "sort_vs_cub": sort_vs_cub,
        "served": served,
        "roofline": roof,
        "frame_roofline": frame_roof,
        "cpu_baseline": cpu,
        "clocks": clocks,
        "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)


def main():
    # a crash in native code prints the Python stack of every thread to stderr
    import faulthandler
    faulthandler.enable(all_threads=True)
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    ap.add_argument("--no-plain", action="store_true", help="skip the single-view leg (profiling runs)")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving leg (profiling runs)")
    ap.add_argument("--no-autotune", action="store_true", help="default knobs (16x16 tiles, 16 views per block)")
    ap.add_argument("--no-ref-cuda", action="store_true",
                    help="skip the reference's own CUDA frame beside the 1024x1024 plain frame")
    ap.add_argument("--only-ref1024", action="store_true",
                    help="time only the reference-compatible 1024x1024 single-view frame (profiling case)")
    ap.add_argument("--views", type=int, default=VIEWS,
                    help="views per batched frame (64 = the workload; fewer only for small profiling cases)")
    args = ap.parse_args()
    globals()["VIEWS"] = args.views
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        if args.impl == "ours":
            torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl" if args.impl == "ours" else "gloo",
                                timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
