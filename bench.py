#!/usr/bin/env python
"""Throughput of the B200 differentiable path tracer on the geometry-gradient workload.

Workload (the reference's headline configuration for fwd+bwd at 512^2): a level-5
icosphere (20,480 triangles, radial vertex noise N(0, 0.02), seed 2, 256^2 texture
seed 0) on a 10x10 ground quad under a 1x1 area light (20,484 triangles in all);
512x512, 32 spp interior, 4 spp primary-edge and 4 spp secondary-edge samples,
max_bounce 3, one light and one BSDF MIS sample. One step = rebuild the scene from
the (translated) vertices, renderD forward, L2 loss against a fixed target, and
the full backward (interior path replay + every boundary term of the estimator).
The default estimator is the unbiased one (its gradient matches central finite
differences; 4 pixel-border samples per border segment); --estimator reference
reproduces the reference's renderD formulas.

Metric: interior path samples (512*512*32 per view) per second of fwd+bwd.
`value` is device time with inputs resident in HBM for the batched step (persistent
scene, rebuild + forward + backward replayed from CUDA graphs); config.other_mode is
the same step through a new Scene and per-view launch sequences. `e2e` adds the
host->device copies of the vertices and texture from pinned memory and the
device->host read of the vertex gradient and the loss, through the public Python
API. `grad_check` compares the translation gradient of sum(w * image) for a smooth
weight image w at the benchmark's sample counts with central differences
(4096-spp renders, common random numbers), outside the timed region.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
Under torchrun every rank renders its own replica (weak scaling, replicas only).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+bwd path samples/s at 512² (batched vs plain) at matched grad error vs FD"
UNIT = "path samples/s"
H = W = 512
SPP = 32
CFG = dict(spp_interior=SPP, spp_primary_edge=4, spp_secondary_edge=4, max_bounce=3, mis_light_samples=1,
           mis_bsdf_samples=1)
WORKLOAD = ("geometry gradient: level-5 icosphere 20,480 tris (+ground, light = 20,484), 512x512, 32 spp interior "
            "+ 4 spp primary edges + 4 spp secondary edges (+ 4 per pixel-border segment, unbiased estimator), "
            "depth 3, L2 loss, fwd+bwd incl. scene rebuild")
TRACE_BYTES_PER_RAY = 40  # ray read 24 B + hit write 16 B (per-ray share of the trace kernel)
# ncu dram__bytes_read.sum + dram__bytes_write.sum of k_trace, mean over the 38 launches of
# one plain step of this workload (2^21-path tiles; ncu flushes the caches before every
# launch, so the BVH is read from DRAM each time), from one capture of
#   ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum,gpu__time_duration.sum -k regex:k_trace -s 12 -c 38
#   python bench.py --mode plain --tile-paths 2097152 --no-autotune --steps 1 --warmup 1 ...
TRACE_DRAM_BYTES_PER_LAUNCH = 72.39e6
TRACE_L2_THROUGHPUT_PCT = (11.9, 14.9)  # ncu lts__throughput, % of peak, 256^2 case
STEP_BYTES_PER_SAMPLE = 2628  # fwd+bwd algorithmic bytes per path sample at depth 3


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def make_spec():
    from torch_psdr_b200 import synth
    return synth.sphere_scene(level=5, tex_hw=256, tex_seed=0, noise_sigma=0.02, noise_seed=2, height=H, width=W)


# ---------------------------------------------------------------- reference (CPU) arm
CPU_BANDS = (4, 16)  # rows of the two bands whose times fix the per-view and per-row costs


def _cpu_band_seconds(orc, spec, rows, seeds):
    """Seconds of one oracle fwd+bwd stand-in on a band of `rows` full-width rows of the
    view: the unbiased estimator's four terms (interior, silhouettes, shadow boundaries,
    pixel borders) evaluated once in forward-mode dual arithmetic (the image value and 8
    directional derivatives per sample, 3 of them the icosphere's translation), including
    the oracle's scene and BVH build. The projection uses cot(fov/2) for both axes, so the
    band subsamples the whole view vertically."""
    import copy
    s = copy.deepcopy(spec)
    s.cameras[0].height = rows
    g = [np.ones((rows, W, 3))]
    t0 = time.perf_counter()
    orc.grad_dir(s, g, which=15, mode=1, seed_verts=seeds, spp_pixel_boundary=4, **CFG)
    return time.perf_counter() - t0


def cpu_rate(spec, seconds_budget=20.0):
    """CPU fwd+bwd path samples/s of the full 512^2 view, all host threads: the oracle's
    step on two row bands gives its per-view cost a (scene build, guiding preprocess) and
    per-row cost b; a full view takes a + 512 b seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc
    orc.lib()
    nthreads = os.cpu_count() or 1
    orc.set_threads(nthreads)
    nv = sum(m.vertices.shape[0] for m in spec.meshes) + sum(l.vertices.shape[0] for l in spec.lights)
    seeds = np.zeros((nv, 3, 8))
    for k in range(3):
        seeds[:spec.meshes[0].vertices.shape[0], k, k] = 1.0
    r1, r2 = CPU_BANDS
    fits = []
    t0 = time.perf_counter()
    while not fits or time.perf_counter() - t0 < seconds_budget:
        t1 = _cpu_band_seconds(orc, spec, r1, seeds)
        t2 = _cpu_band_seconds(orc, spec, r2, seeds)
        b = max(t2 - t1, 1e-9) / (r2 - r1)
        fits.append((t1 - b * r1, b))
    a = statistics.median(f[0] for f in fits)
    b = statistics.median(f[1] for f in fits)
    full = a + b * H
    sample = (f"oracle fwd+bwd stand-in: the unbiased estimator's interior, silhouette, shadow-boundary and "
              f"pixel-border terms in forward-mode duals (image + 8 directional derivatives) at the benchmark's "
              f"sample counts, on bands of {r1} and {r2} rows x {W}; per view {a:.3f} s + {b * 1e3:.2f} ms per row "
              f"-> {full:.2f} s for the full {H}x{W} view (median of {len(fits)} band pairs in "
              f"{time.perf_counter() - t0:.1f} s)")
    return H * W * SPP / full, nthreads, sample, full


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    spec = make_spec()
    for _ in range(args.warmup):
        cpu_rate(spec, seconds_budget=0.0)
    vals, cores, sample, step_s = [], 1, "", []
    for _ in range(args.steps):
        v, cores, sample, full = cpu_rate(spec, seconds_budget=0.0)
        vals.append(v)
        step_s.append(full)
    value = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(step_s),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64 duals (f32 geometry)",
            "data": "synthetic (seeded icosphere scene)", "config": {"workload": WORKLOAD},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- clocks
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, dev_index):
        self.p = None
        self.dev = dev_index
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(dev_index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                      stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        out, _ = self.p.communicate(timeout=10)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- gradient check
def smooth_weights(torch, dev):
    yy, xx = torch.meshgrid(torch.arange(H, device=dev) + 0.5, torch.arange(W, device=dev) + 0.5, indexing="ij")
    return torch.stack([torch.sin(2 * math.pi * xx / W * 1.3 + c) * torch.cos(2 * math.pi * yy / H * 0.7) + 0.3
                        for c in range(3)], -1).float().contiguous()


def grad_check(torch, dr, integ, build_scene, base, tex, dev, h=1e-3, fd_spp=4096, replicas=4, ad_replicas=16):
    """Translation gradient of Phi = sum(w * image) for a smooth weight image w, from the
    estimator at the benchmark's sample counts, against central differences of Phi from
    fd_spp-spp renders (same sample streams at +-h). The estimator is averaged over
    `ad_replicas` independent sample streams (seeds 1..ad_replicas; one step's gradient
    costs a benchmark step), the finite differences over `replicas`; the spreads give the
    standard error of each mean and the spread of a single step's gradient. The
    benchmark's own L2 loss is not used here: its image gradient is dominated by
    texel-scale residuals, which makes its finite differences ill-conditioned (they move by
    tens of percent with h and spp)."""
    from torch_psdr_b200 import _lib as L
    w = smooth_weights(torch, dev)
    wd = w.double()
    kw = {k: getattr(integ.cfg, k) for k in ("spp_interior", "spp_primary_edge", "spp_secondary_edge",
                                              "spp_pixel_boundary", "max_bounce")}
    est = "unbiased" if integ.cfg.estimator == L.EST_UNBIASED else "reference"
    ads, fds = [], []
    for r in range(1, ad_replicas + 1):
        ad_integ = dr.PathIntegrator(estimator=est, seed=r, **kw)
        t = torch.zeros(3, device=dev, requires_grad=True)
        ad_integ.renderD(build_scene(base + t, tex))[0].backward(w)
        ads.append(t.grad.double().cpu().numpy())
    for r in range(1, replicas + 1):
        fd_integ = dr.PathIntegrator(**dict(CFG, spp_interior=fd_spp, seed=r))
        fd = []
        with torch.no_grad():
            for k in range(3):
                e = torch.zeros(3, device=dev)
                e[k] = h
                lp = float((fd_integ.renderC(build_scene(base + e, tex))[0].double() * wd).sum())
                lm = float((fd_integ.renderC(build_scene(base - e, tex))[0].double() * wd).sum())
                fd.append((lp - lm) / (2 * h))
        fds.append(np.array(fd))
    ads, fds = np.array(ads), np.array(fds)
    ad, fd = ads.mean(0), fds.mean(0)
    se = lambda a: a.std(0, ddof=1) / np.sqrt(len(a)) if len(a) > 1 else np.zeros(3)
    single = np.array([np.linalg.norm(a - fd) / np.linalg.norm(fd) for a in ads])
    return {"rel_l2_vs_fd": float(np.linalg.norm(ad - fd) / np.linalg.norm(fd)), "ad": ad.tolist(), "fd": fd.tolist(),
            "ad_stderr": se(ads).tolist(), "fd_stderr": se(fds).tolist(),
            "rel_l2_fd_stderr": float(np.linalg.norm(se(fds)) / np.linalg.norm(fd)),
            "rel_l2_ad_stderr": float(np.linalg.norm(se(ads)) / np.linalg.norm(fd)),
            "single_step_rel_l2_median": float(np.median(single)), "ad_replicas": ad_replicas,
            "functional": "sum(w * image), w = sin(2.6 pi x/W + c) cos(1.4 pi y/H) + 0.3 per channel c",
            "parameter": "translation of the icosphere", "estimator": est,
            "fd_step": h, "fd_spp": fd_spp, "replicas": replicas, "seeds": list(range(1, max(replicas, ad_replicas) + 1))}


# ---------------------------------------------------------------- per-phase breakdown
TERMS = ((1, "interior"), (2, "silhouettes"), (4, "shadow_boundaries"), (8, "pixel_borders"),
         (64, "indirect_shadow_boundaries"), (32, "creases"))


def phase_breakdown(torch, dr, integ_kw, run_step, flush, reps=3):
    """Device milliseconds of the plain step's phases, each timed alone with CUDA events
    (median of `reps` after one warm-up, L2 flushed before each): `forward` = scene
    construction + renderD forward + loss with the backward skipped; each gradient term =
    a plain step whose backward is restricted to that term (gradient_terms), minus
    `forward`. run_step(integ, backward) runs one plain step."""
    stream = torch.cuda.current_stream()

    def med(fn):
        ts = []
        for r in range(reps + 1):
            flush.fill_(float(r))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize()
            if r:
                ts.append(a.elapsed_time(b))
        return statistics.median(ts)

    base = dr.PathIntegrator(**integ_kw)
    fwd = med(lambda: run_step(base, False))
    out = {"forward": fwd}
    total = fwd
    est = integ_kw.get("estimator", "reference")
    for bit, name in TERMS:
        if est != "unbiased" and bit not in (1, 2, 4):
            continue
        integ = dr.PathIntegrator(**dict(integ_kw, gradient_terms=bit))
        t = max(0.0, med(lambda: run_step(integ, True)) - fwd)
        out[name] = t
        total += t
    out["sum"] = total
    return out


# ---------------------------------------------------------------- replicas
def max_over_ranks(value, dist, device):
    """The largest of the ranks' values (device times are taken as the max over ranks);
    the value itself on one process (dist None)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, units_per_rank_step, steps, ms):
    """Whole-job throughput of `world` replicas that each processed units_per_rank_step
    units per step for `steps` steps in `ms` milliseconds (the max over ranks)."""
    return world * units_per_rank_step * steps / (ms / 1e3)


# ---------------------------------------------------------------- B200 arm
def run_b200(args):
    import torch
    import torch_psdr_b200 as dr
    from torch_psdr_b200 import _lib as L

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as tdist
        from datetime import timedelta
        tdist.init_process_group("nccl", timeout=timedelta(seconds=300))
        dist = tdist
    dev = torch.device("cuda", local)
    lib = L.load()
    spec = make_spec()
    sphere, ground = spec.meshes
    light = spec.lights[0]
    c = spec.cameras[0]

    def tens(a, dt=torch.float32, rg=False):
        return torch.tensor(np.asarray(a), dtype=dt, device=dev, requires_grad=rg)

    base = tens(sphere.vertices)
    faces = tens(sphere.faces, torch.int32)
    uvs, uvi = tens(sphere.uvs), tens(sphere.uv_indices, torch.int32)
    tex = tens(sphere.texture)
    gV, gF, gT = tens(ground.vertices), tens(ground.faces, torch.int32), tens(ground.texture)
    lV, lF, lE = tens(light.vertices), tens(light.faces, torch.int32), tens(light.emit)
    cam = dr.PerspectiveCamera(tens(c.look_from), tens(c.look_at), tens(c.up), tens([c.vfov]), H, W)
    integ = dr.PathIntegrator(estimator=args.estimator, batch_lanes=args.batch_lanes,
                              batch_records=args.batch_records, tile_paths=args.tile_paths, **CFG)

    leaf = {"size": 1}

    def build_scene(verts, texture):
        sc = dr.Scene([cam], [dr.Mesh(verts, uvs, faces, uvi, dr.DiffuseMaterial(texture)),
                              dr.Mesh(gV, None, gF, None, dr.DiffuseMaterial(gT))],
                      [dr.AreaLight(lV, lF, lE)])
        if leaf["size"] != 1:
            L.check(lib.psdr_scene_set_leaf_size(sc.handle, leaf["size"],
                                                 ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)), "leaf")
        return sc

    # tile size (and leaf size, kept per scene) from the library's autotuner, untimed
    tune = integ.autotune(build_scene(base, tex)) if not args.no_autotune else None
    if tune:
        leaf["size"] = tune["leaf_size"]
    with torch.no_grad():
        target = integ.renderC(build_scene(base + torch.tensor([0.05, 0.0, 0.0], device=dev), tex))[0].clone()
    t = torch.zeros(3, device=dev, requires_grad=True)

    def step_plain(verts_base, texture):
        # the reference's usage: a new Scene per optimisation step, renderD, loss, backward
        if t.grad is not None:
            t.grad = None
        v = verts_base + t
        scene = build_scene(v, texture)
        img = integ.renderD(scene)[0]
        loss = ((img - target) ** 2).sum()
        loss.backward()
        return loss

    batch_state = {}

    def step_batched(verts_base, texture):
        # one persistent scene + BatchRender: geometry rebuild and render replayed from a graph
        if t.grad is not None:
            t.grad = None
        v = verts_base + t
        if "batch" not in batch_state:
            sc = build_scene(v, texture)
            batch_state["scene"] = sc
            batch_state["batch"] = dr.BatchRender(integ, [sc])
        sc = batch_state["scene"]
        sc.meshes[0].set_vertices(v)
        if texture.data_ptr() != sc.meshes[0].material.texture.data.data_ptr():
            sc.meshes[0].material.texture.data.copy_(texture)
        img = batch_state["batch"].renderD()[0]
        loss = ((img - target) ** 2).sum()
        loss.backward()
        return loss

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()

    def timed(stepfn, with_clocks):
        """Device time (ms, summed over the timed steps, max over ranks) plus the
        in-library profile of the timed region."""
        L.check(lib.psdr_profile_enable(1), "profile")  # before warm-up: graphs record their trace events
        for _ in range(args.warmup):
            stepfn(base, tex)
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        L.check(lib.psdr_profile_reset(), "profile")
        clocks = Clocks(local) if with_clocks else None
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.fill_(float(k))  # evicts L2 between steps, outside the timed events
            ev[k][0].record(stream)
            stepfn(base, tex)
            ev[k][1].record(stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        clk = clocks.stop() if clocks else None
        total = sum(a.elapsed_time(b) for a, b in ev)
        prof = (ctypes.c_int64 * 3)()
        tms = ctypes.c_double()
        L.check(lib.psdr_profile_read(prof, ctypes.byref(tms)), "profile")
        L.check(lib.psdr_profile_enable(0), "profile")
        total = max_over_ranks(total, dist, dev)
        return total, (int(prof[0]), int(prof[1]), int(prof[2])), tms.value, clk

    samples = H * W * SPP
    step = step_batched if args.mode == "batched" else step_plain
    other = step_plain if args.mode == "batched" else step_batched
    total_ms, (launches, trace_launches, rays), trace_ms_v, clk = timed(step, True)
    value = job_rate(world, samples, args.steps, total_ms)
    other_ms, other_prof, other_trace_ms, _ = timed(other, False)
    # the trace kernel's launch durations for the roofline come from the plain step, whose
    # launches run one at a time (the batched graph overlaps kernels of concurrent lanes)
    if args.mode == "plain":
        plain_ms, (_, plain_tl, plain_rays), plain_trace_ms = total_ms, (launches, trace_launches, rays), trace_ms_v
    else:
        plain_ms, (_, plain_tl, plain_rays), plain_trace_ms = other_ms, other_prof, other_trace_ms
    other_value = job_rate(world, samples, args.steps, other_ms)

    # ---------------- end-to-end through the public API with host buffers
    h_base = torch.tensor(sphere.vertices, dtype=torch.float32).pin_memory()
    h_tex = torch.tensor(sphere.texture, dtype=torch.float32).pin_memory()
    h_grad = torch.empty((sphere.vertices.shape[0], 3), dtype=torch.float32).pin_memory()
    h_loss = torch.empty((), dtype=torch.float32).pin_memory()
    vb = torch.empty_like(base)
    vt = torch.empty_like(tex)

    def e2e_step():
        vb.copy_(h_base, non_blocking=True)
        vt.copy_(h_tex, non_blocking=True)
        vv = vb.detach().requires_grad_(True)
        loss = step(vv, vt)
        h_grad.copy_(vv.grad, non_blocking=True)
        h_loss.copy_(loss.detach(), non_blocking=True)

    e2e_step()
    torch.cuda.synchronize()
    ee = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    for k in range(args.steps):
        flush.fill_(float(k))
        ee[k][0].record(stream)
        e2e_step()
        ee[k][1].record(stream)
    torch.cuda.synchronize()
    e2e_ms = sum(a.elapsed_time(b) for a, b in ee)
    e2e_ms = max_over_ranks(e2e_ms, dist, dev)
    e2e_value = job_rate(world, samples, args.steps, e2e_ms)
    h2d = h_base.numel() * 4 + h_tex.numel() * 4
    d2h = h_grad.numel() * 4 + 4

    peak, peak_kind = peaks()
    trace_avg_ms = plain_trace_ms / max(1, plain_tl)
    achieved = (plain_rays / max(1, plain_tl)) * TRACE_BYTES_PER_RAY / (trace_avg_ms / 1e3) / 1e9
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded icosphere scene)",
            "config": {"workload": WORKLOAD,
                       "mode": ("batched (persistent scene, geometry rebuild + fwd and bwd replayed from CUDA graphs)"
                                if args.mode == "batched" else "plain (new Scene per step, per-view launch sequences)"),
                       "estimator": args.estimator,
                       "autotune": tune,
                       "other_mode": {"mode": "plain" if args.mode == "batched" else "batched",
                                      "value": other_value, "ms_per_step": other_ms / args.steps},
                       "l2": "flushed between steps (256 MiB write outside the timed events)",
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "kernel": "k_trace (LBVH closest hit)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "traffic": TRACE_DRAM_BYTES_PER_LAUNCH,
                         "traffic_source": "ncu DRAM bytes per k_trace launch, mean over the 38 launches of "
                                           "one plain step at 2^21-path tiles (caches flushed per launch)",
                         "l2_throughput_pct_of_peak_ncu": list(TRACE_L2_THROUGHPUT_PCT),
                         "bytes_per_unit": f"{TRACE_BYTES_PER_RAY} B/ray",
                         "rays_per_launch": plain_rays / max(1, plain_tl), "avg_launch_ms": trace_avg_ms,
                         "timed_in": "plain step (launches one at a time)",
                         "trace_share_of_step": plain_trace_ms / max(plain_ms, 1e-9),
                         "step_algorithmic_gbs": samples * STEP_BYTES_PER_SAMPLE / (total_ms / args.steps / 1e3) / 1e9},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches, "clocks": clk,
            "rays_per_s": rays / (total_ms / 1e3)}
    if rank == 0 and world == 1 and not args.no_phases:
        integ_kw = dict(CFG, estimator=args.estimator, tile_paths=int(integ.cfg.tile_paths),
                        trace_queue=int(integ.cfg.trace_queue))

        def run_phase_step(pi, backward):
            tt = torch.zeros(3, device=dev, requires_grad=backward)
            img = pi.renderD(build_scene(base + tt, tex))[0]
            loss = ((img - target) ** 2).sum()
            if backward:
                loss.backward()

        line["config"]["phases_ms"] = phase_breakdown(torch, dr, integ_kw, run_phase_step, flush)
    if rank == 0 and world == 1 and not args.no_grad_check:
        try:
            line["grad_check"] = grad_check(torch, dr, integ, build_scene, base, tex, dev)
        except Exception as exc:  # the measured line is printed either way
            line["grad_check"] = {"error": f"{type(exc).__name__}: {exc}"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, cores, sample, _ = cpu_rate(spec, seconds_budget=20.0)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------- multi-view workload
MV_WORKLOAD = ("multi-view geometry + texture gradient: 64 views, H and W ~ U{128..512} (seed 3) on the radius-4 "
               "sphere, over 3 scenes (geodesic spheres of 5,120 / 50,000 / 200,000 tris, noise 0.02, 256^2 texture, "
               "ground, light), view v on scene v mod 3, 16 spp interior + 4 spp per edge kind, depth 4, L2 loss")


def run_multiview(args):
    """Batched (one work list and one graph each way for all 64 views) against plain
    (per view: a new single-camera Scene, renderD, loss, backward), one GPU."""
    import torch
    import torch_psdr_b200 as dr
    from torch_psdr_b200 import synth
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    cams = synth.orbit_cameras(64, 4.0, seed=3, size_lo=128, size_hi=512)
    cfg = dict(spp_interior=16, spp_primary_edge=4, spp_secondary_edge=4, max_bounce=4, estimator=args.estimator)
    integ = dr.PathIntegrator(batch_lanes=args.batch_lanes, batch_records=args.batch_records, **cfg)

    def tens(a, dt=torch.float32, rg=False):
        return torch.tensor(np.asarray(a), dtype=dt, device=dev, requires_grad=rg)

    scenes_data = []
    for i, n in enumerate((16, 50, 100)):
        spec = synth.sphere_scene(freq=n, tex_hw=256, tex_seed=i, noise_sigma=0.02, noise_seed=2)
        sph, gr = spec.meshes
        lt = spec.lights[0]
        d = dict(v=tens(sph.vertices, rg=True), f=tens(sph.faces, torch.int32), uv=tens(sph.uvs),
                 uvi=tens(sph.uv_indices, torch.int32), tex=tens(sph.texture, rg=True), gV=tens(gr.vertices),
                 gF=tens(gr.faces, torch.int32), gT=tens(gr.texture), lV=tens(lt.vertices),
                 lF=tens(lt.faces, torch.int32), lE=tens(lt.emit))
        d["cams"] = [dr.PerspectiveCamera(tens(c.look_from), tens(c.look_at), tens(c.up), tens([c.vfov]), c.height,
                                          c.width) for k, c in enumerate(cams) if k % 3 == i]
        scenes_data.append(d)

    def scene_of(d, cam_list, verts=None):
        return dr.Scene(cam_list, [dr.Mesh(d["v"] if verts is None else verts, d["uv"], d["f"], d["uvi"],
                                           dr.DiffuseMaterial(d["tex"])),
                                   dr.Mesh(d["gV"], None, d["gF"], None, dr.DiffuseMaterial(d["gT"]))],
                        [dr.AreaLight(d["lV"], d["lF"], d["lE"])])

    with torch.no_grad():
        targets = [[img.clone() for img in integ.renderC(scene_of(d, d["cams"], d["v"] + 0.03))] for d in scenes_data]
    views = sum(len(d["cams"]) for d in scenes_data)
    paths = sum(c.height * c.width for c in cams) * cfg["spp_interior"]

    def step_plain():
        for d, tg in zip(scenes_data, targets):
            for cam, t in zip(d["cams"], tg):
                img = integ.renderD(scene_of(d, [cam]))[0]
                ((img - t) ** 2).sum().backward()

    batch_scenes = [scene_of(d, d["cams"]) for d in scenes_data]
    batch = dr.BatchRender(integ, batch_scenes)
    flat_targets = [t for tg in targets for t in tg]

    def step_batched():
        imgs = batch.renderD()
        sum(((a - b) ** 2).sum() for a, b in zip(imgs, flat_targets)).backward()

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()

    def timed(fn, with_clocks):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        clocks = Clocks(dev.index) if with_clocks else None
        for k in range(args.steps):
            flush.fill_(float(k))
            ev[k][0].record(stream)
            fn()
            ev[k][1].record(stream)
        torch.cuda.synchronize()
        clk = clocks.stop() if clocks else None
        return sum(a.elapsed_time(b) for a, b in ev), clk

    b_ms, clk = timed(step_batched, True)
    p_ms, _ = timed(step_plain, False)
    phases = None
    if not args.no_phases:
        def run_phase_step(pi, backward):
            for d, tg in zip(scenes_data, targets):
                for cam, t in zip(d["cams"], tg):
                    img = pi.renderD(scene_of(d, [cam]))[0]
                    loss = ((img - t) ** 2).sum()
                    if backward:
                        loss.backward()

        phases = phase_breakdown(torch, dr, cfg, run_phase_step, flush, reps=3)
    value = paths * args.steps / (b_ms / 1e3)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": b_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded geodesic-sphere scenes, orbit cameras)",
            "config": {"workload": MV_WORKLOAD, "views": views, "paths_per_step": paths, "estimator": args.estimator,
                       "mode": "batched (one work list, forward and backward graphs)",
                       "other_mode": {"mode": "plain (per view: new Scene, renderD, backward)",
                                      "value": paths * args.steps / (p_ms / 1e3), "ms_per_step": p_ms / args.steps},
                       "batched_over_plain": p_ms / b_ms, "phases_ms": phases,
                       "l2": "flushed between steps (256 MiB write outside the timed events)"},
            "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- large workload
LG_WORKLOAD = ("large scene, full gradient with path replay: 16 noisy level-6 icospheres (1,310,720 tris) centred "
               "uniformly in [-5,5]^3 (seed 4), a 512^2 texture each, ground, 4x4 light; 1024x1024, 64 spp interior "
               "+ 4 spp per edge kind, depth 5, vertex + texture gradients of an L2 loss")


def run_large(args):
    """One persistent Scene of 16 level-6 spheres rendered and differentiated through
    BatchRender (forward and backward replayed from graphs), one GPU."""
    import torch
    import torch_psdr_b200 as dr
    from torch_psdr_b200 import synth
    t0 = time.time()
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    spec = synth.large_scene()
    cfg = dict(spp_interior=64, spp_primary_edge=4, spp_secondary_edge=4, max_bounce=5, estimator=args.estimator)
    integ = dr.PathIntegrator(batch_lanes=args.batch_lanes, batch_records=args.batch_records, **cfg)

    def tens(a, dt=torch.float32, rg=False):
        return torch.tensor(np.asarray(a), dtype=dt, device=dev, requires_grad=rg)

    spheres, ground = spec.meshes[:-1], spec.meshes[-1]
    sv = [tens(m.vertices, rg=True) for m in spheres]
    st = [tens(m.texture, rg=True) for m in spheres]
    f, uv, uvi = tens(spheres[0].faces, torch.int32), tens(spheres[0].uvs), tens(spheres[0].uv_indices, torch.int32)
    gV, gF, gT = tens(ground.vertices), tens(ground.faces, torch.int32), tens(ground.texture)
    lt, c = spec.lights[0], spec.cameras[0]
    light = dr.AreaLight(tens(lt.vertices), tens(lt.faces, torch.int32), tens(lt.emit))
    cam = dr.PerspectiveCamera(tens(c.look_from), tens(c.look_at), tens(c.up), tens([c.vfov]), c.height, c.width)

    def scene_of(verts):
        return dr.Scene([cam], [dr.Mesh(v, uv, f, uvi, dr.DiffuseMaterial(t)) for v, t in zip(verts, st)] +
                        [dr.Mesh(gV, None, gF, None, dr.DiffuseMaterial(gT))], [light])

    with torch.no_grad():
        target = integ.renderC(scene_of([v + 0.03 for v in sv]))[0].clone()
    batch = dr.BatchRender(integ, [scene_of(sv)])
    print(f"large: setup {time.time() - t0:.1f} s", file=sys.stderr, flush=True)

    def step():
        img = batch.renderD()[0]
        ((img - target) ** 2).sum().backward()

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    print(f"large: warm-up done {time.time() - t0:.1f} s", file=sys.stderr, flush=True)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clocks = Clocks(dev.index)
    for k in range(args.steps):
        flush.fill_(float(k))
        ev[k][0].record(stream)
        step()
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = sum(a.elapsed_time(b) for a, b in ev)
    paths = c.height * c.width * cfg["spp_interior"]
    g = sv[0].grad
    line = {"metric": METRIC, "value": paths * args.steps / (ms / 1e3), "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded icosphere scene)",
            "config": {"workload": LG_WORKLOAD, "triangles": sum(len(m.faces) for m in spec.meshes) + len(lt.faces),
                       "paths_per_step": paths, "estimator": args.estimator,
                       "mode": "batched (persistent scene, forward and backward graphs)",
                       "l2": "flushed between steps (256 MiB write outside the timed events)",
                       "grad_finite": bool(torch.isfinite(g).all().item()) and float(g.abs().sum()) > 0},
            "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference", "ours"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-grad-check", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-phases", action="store_true", help="skip the per-phase breakdown of the plain step")
    ap.add_argument("--tile-paths", type=int, default=0,
                    help="wavefront tile (paths; 0 = library default, or the autotuner's pick)")
    ap.add_argument("--batch-lanes", type=int, default=0, help="PathIntegrator batch_lanes (0 = library default)")
    ap.add_argument("--batch-records", type=int, default=0, choices=[-1, 0, 1],
                    help="PathIntegrator batch_records (0 = keep when they fit a quarter of free memory)")
    ap.add_argument("--estimator", default="unbiased", choices=["unbiased", "reference"])
    ap.add_argument("--workload", default="geometry", choices=["geometry", "multiview", "large"],
                    help="geometry: the 512^2 fwd+bwd workload (default); multiview: 64 views over 3 scenes; "
                         "large: 16 level-6 spheres at 1024^2, 64 spp, depth 5")
    ap.add_argument("--mode", default="batched", choices=["batched", "plain"],
                    help="batched: persistent scene + graph replay; plain: new Scene + per-view launches each step")
    ap.add_argument("--size", type=int, default=512, help="image size (512 = the benchmark workload)")
    ap.add_argument("--spp", type=int, default=32, help="interior spp (32 = the benchmark workload)")
    args = ap.parse_args()
    global H, W, SPP
    if args.size != 512 or args.spp != 32:
        H = W = args.size
        SPP = args.spp
        CFG["spp_interior"] = SPP
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "multiview":
        return run_multiview(args)
    if args.workload == "large":
        return run_large(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
