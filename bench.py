"""Benchmark of the differentiable render path on one B200 (render-only kernel benchmark
configuration): 1,000,000 Gaussians, one 1920x1080 view, plain FP32 forward and backward
with an upstream dL/dpixel drawn N(0,1) per channel. The compositing configuration (tile
shape x chunk depth) is autotuned on this workload before warm-up (--raster fixes one).

One step = projection + binning (scan, key emission, radix sort, tile ranges) +
compositing forward + compositing backward + projection backward for that view. The metric
is megapixels per second of forward+backward (W*H per step). Inputs are larger than L2 (the
parameter planes alone are 240 MB), so no L2 flush is needed between steps.

Usage:
  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Under torchrun every rank runs an independent replica of the workload (the path does not
shard across views in this configuration); the slowest rank's time is reported.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WIDTH, HEIGHT = 1920, 1080
METRIC = "train iters/s and Mpix/s fwd+bwd at 1 B200 vs plain GPU & CPU, at matched PSNR"
UNIT = "Mpix/s"
WORKLOAD = "render fwd+bwd, 1M Gaussians, 1920x1080, SH degree 3, dL/dpix ~ N(0,1)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--cpu-steps", type=int, default=3, help="steps of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--raster", default="auto",
                    help="compositing configuration: 'auto' (autotune) or TWxTHxCHUNK[/PIXELS_PER_THREAD], "
                         "e.g. 16x16x256/2")
    ap.add_argument("--no-train", action="store_true", help="skip the small-scene training run (10k-Gaussian blobs, 256x256 views)")
    ap.add_argument("--no-train-shells", action="store_true",
                    help="skip plain training on the clustered 500k-Gaussian multi-view scene (30,000 iterations) "
                         "and its CPU samples")
    ap.add_argument("--train-shells-iters", type=int, default=0, help="iterations of that run (default: all 30,000)")
    ap.add_argument("--shells-cpu-iters", type=int, default=3,
                    help="timed CPU oracle iterations at each sampled model state of that run")
    ap.add_argument("--train-batched", action="store_true",
                    help="batched mixed-size BF16 training on the same scene (8 views per step)")
    ap.add_argument("--train-batched-iters", type=int, default=0, help="steps of that run (default: all 3,750)")
    ap.add_argument("--train-learned", action="store_true",
                    help="learned densification: learn on scene seeds 2-5, compare with the rule on seed 6")
    ap.add_argument("--learn-iters", type=int, default=1875, help="steps of each learning run")
    ap.add_argument("--no-train-target", action="store_true",
                    help="skip the training-target comparison (plain one-view trainer vs the batched, coarse-to-fine, "
                         "learned-densification trainer on the clustered scene)")
    ap.add_argument("--profile-mlp", action="store_true",
                    help="only the densification network's forward (tcgen05) on 4M rows, for an ncu capture")
    ap.add_argument("--mlp-rows", type=int, default=4_000_000)
    ap.add_argument("--profile-train", action="store_true",
                    help="only a short shell-scene training run (20 views, 300 iterations) for an ncu launch list; "
                         "prints the launches before its last 100 iterations")
    ap.add_argument("--profile-blobs", action="store_true",
                    help="only a short blob-scene training run (300 iterations, densification from 100 every 100) for "
                         "an ncu launch list; prints the launches before its last 100 iterations")
    ap.add_argument("--profile-small", action="store_true",
                    help="a reduced case for ncu captures (fewer Gaussians, one step)")
    ap.add_argument("--profile-stages", action="store_true",
                    help="only the HBM-bound stages, twice each, for an ncu capture: projection forward and backward "
                         "and Adam over 1M Gaussians, the SSIM + L1 loss on one 1297x840 view")
    return ap.parse_args()


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_first(self, timeout=2.0):
        """Until the first sample arrives (or `timeout` s)."""
        t0 = time.time()
        while self.proc is not None and not self.lines and time.time() - t0 < timeout:
            time.sleep(0.01)

    def wait_next(self, timeout=2.0):
        """Until one more sample arrives after this call (so the window closes after the
        region it brackets)."""
        n, t0 = len(self.lines), time.time()
        while self.proc is not None and len(self.lines) <= n and time.time() - t0 < timeout:
            time.sleep(0.01)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(value: float, world: int, device=None) -> float:
    """The slowest rank's value (every rank calls this in the same order)."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def unit_peaks(ctx, local):
    """FP32 (FMA) and special-function-unit (ex2) throughput measured on this GPU by the
    library's microbenchmark (splat_diag_peak), best of three, with the SM clock sampled
    while it runs: the denominators of the compositing stages' roofline."""
    sampler = ClockSampler(local)
    sampler.start()
    fp32 = max(ctx.peak("fp32")["ops_per_s"] for _ in range(3))
    mufu = max(ctx.peak("mufu")["ops_per_s"] for _ in range(3))
    clocks = sampler.stop()
    return {"fp32_tflops": round(fp32 / 1e12, 2), "mufu_gops": round(mufu / 1e9, 1),
            "source": "measured (splat_diag_peak: FMA and ex2 chains on every SM, CUDA events)",
            "clocks": clocks}


# Algorithmic work per unit (fixed constants): bytes for the HBM-bound stages.
PROJ_FWD_BYTES = 236 + 64          # parameters read + projection record written, per Gaussian
PROJ_BWD_BYTES = 236 + 36 + 236    # parameters + screen gradients read, parameter gradients written
SORT_BYTES_PER_KEY_PASS = 24       # one read and one write of a (u64 key, u32 value) pair
EMIT_BYTES_PER_ENTRY = 12          # key + value written
RASTER_FWD_BYTES_PER_PIXEL = 20    # image (12) + final T (4) + n_contrib (4) written
RASTER_BWD_BYTES_PER_PIXEL = 20    # dL/dpix (12) + final T (4) + n_contrib (4) read
RASTER_BYTES_PER_ENTRY = 52        # sorted index (4) + record gather (48)
# dram__bytes_read.sum + dram__bytes_write.sum per launch, ncu, default workload.
NCU_DRAM_BYTES_1M = {("raster_bwd", 16, 16, 256, 1): int((197.05 + 17.84) * 1e6),
                     ("raster_fwd", 16, 16, 256, 1): int((82.84 + 20.76) * 1e6),
                     ("raster_bwd", 16, 16, 128, 2): int((196.84 + 17.58) * 1e6),
                     ("raster_fwd", 16, 16, 128, 2): int((82.91 + 21.21) * 1e6),
                     ("raster_bwd", 16, 16, 256, 2): int((196.72 + 16.80) * 1e6),
                     ("raster_fwd", 16, 16, 256, 2): int((82.95 + 22.06) * 1e6),
                     ("raster_bwd", 16, 32, 256, 2): int((185.54 + 13.20) * 1e6),
                     ("raster_fwd", 16, 32, 256, 2): int((74.59 + 16.79) * 1e6)}
RASTER_FWD_FLOP_PER_PAIR = 20
RASTER_BWD_FLOP_PER_PAIR = 50
RASTER_FWD_SFU_PER_PAIR = 1        # one exp
RASTER_BWD_SFU_PER_PAIR = 2        # one exp, one reciprocal (the transmittance division)
BIN_BYTES_PER_ENTRY = 40 + 24      # key emission (key 8 + value 4 + entry Gaussian 4, Proj read) + sort (24)


def stage_rooflines(stage_ms, n, entries, pairs_fwd, pairs_bwd, pixels, hbm_gbs, fp32_tflops, mufu_gops):
    """Per stage: the algorithmic work, the time each unit's peak needs for it, the bound
    (the unit needing the longest) and the fraction of that bound achieved."""
    work = {
        "project_fwd": {"bytes": PROJ_FWD_BYTES * n},
        "bin": {"bytes": BIN_BYTES_PER_ENTRY * entries},
        "raster_fwd": {"bytes": RASTER_FWD_BYTES_PER_PIXEL * pixels + RASTER_BYTES_PER_ENTRY * entries,
                       "flop": RASTER_FWD_FLOP_PER_PAIR * pairs_fwd, "sfu": RASTER_FWD_SFU_PER_PAIR * pairs_fwd},
        "raster_bwd": {"bytes": RASTER_BWD_BYTES_PER_PIXEL * pixels + RASTER_BYTES_PER_ENTRY * entries,
                       "flop": RASTER_BWD_FLOP_PER_PAIR * pairs_bwd, "sfu": RASTER_BWD_SFU_PER_PAIR * pairs_bwd},
        "project_bwd": {"bytes": PROJ_BWD_BYTES * n},
    }
    out = {}
    for k, w in work.items():
        t = {"hbm": w["bytes"] / (hbm_gbs * 1e9) * 1e3}
        if "flop" in w:
            t["fp32"] = w["flop"] / (fp32_tflops * 1e12) * 1e3
            t["mufu"] = w["sfu"] / (mufu_gops * 1e9) * 1e3
        bound = max(t, key=t.get)
        out[k] = {**w, "ms": round(stage_ms[k], 4), "roofline_ms": round(t[bound], 4), "bound": bound,
                  "frac": round(t[bound] / stage_ms[k], 4), "unit_ms": {u: round(v, 4) for u, v in t.items()}}
    return out


REF_MAX_STEPS, REF_MAX_WARMUP = 200, 20


def workload_config(n, world):
    """The workload's `config`, the same in both arms."""
    return {"workload": WORKLOAD, "gaussians": n, "width": WIDTH, "height": HEIGHT,
            "l2": "inputs larger than L2 (240 MB parameter planes), no flush", "parallelism": f"replicas x{world}"}


def run_ours(args, rank, world, local):
    import torch
    from splatrs_b200 import gpu as G
    from splatrs_b200 import scenes
    from splatrs_b200._lib import Camera, ProjOpts

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.n
    s = scenes.render_benchmark_scene(n=n)
    cam = Camera.from_record(s["cam"])
    opts = ProjOpts.make(sh_degree=3)
    bg = s["background"]
    stream = torch.cuda.current_stream(dev)
    ctx = G.Context(local, stream)

    params = torch.from_numpy(s["params"]).to(dev)
    planes = G.params_to_planes(ctx, params)
    dimage = torch.from_numpy(s["dimage"]).to(dev)
    pgrad = torch.zeros((3, n, 4), dtype=torch.float32, device=dev)
    del params

    peaks = unit_peaks(ctx, local)

    # Compositing configuration: every candidate timed on this workload, the fastest kept.
    tuning = None
    if args.raster == "auto":
        tuning = ctx.autotune_render(planes, n, n, cam, opts, bg, dimage, reps=3)
        tuning = {"picked": list(tuning["picked"]),
                  "ms_per_pass": {f"{a}x{b}x{c}/{d}": round(v, 4) for (a, b, c, d), v in tuning["ms"].items()}}
    else:
        ctx.raster_config = tuple(int(v) for v in args.raster.replace("/", "x").split("x"))
    raster = ctx.raster_config

    # Stage-level step with events between stages.
    def full_step(ev=None):
        def mark(i):
            if ev is not None:
                ev[i].record(stream)
        mark(0)
        proj = G.project_all(ctx, planes, n, n, cam, opts)
        mark(1)
        b = G.bin(ctx, proj)
        mark(2)
        out = G.rasterize_forward(ctx, proj, b, bg, count_pairs=ev is None)
        mark(3)
        ctx.zero(pgrad)
        G.rasterize_backward(ctx, proj, b, bg, out, dimage, pgrad=pgrad, cap=n)
        mark(4)
        G.project_backward_all(ctx, planes, n, n, cam, opts, proj, pgrad)
        mark(5)
        return proj, b, out

    # Counters from one untimed step: entries, pairs.
    proj, b, out = full_step()
    pairs_fwd = int(out.pairs.item())
    pp = torch.zeros(1, dtype=torch.int64, device=dev)
    ctx.zero(pgrad)
    G.rasterize_backward(ctx, proj, b, bg, out, dimage, pgrad=pgrad, cap=n, pairs=pp)
    pairs_bwd = int(pp.item())
    entries = b.num_entries
    visible = int((proj.num_tiles > 0).sum().item())
    torch.cuda.synchronize(dev)

    # nvidia-smi samples every 100 ms, longer than the timed steps take: the sampler runs
    # from before the warm-up to after the timed region, and waits for its first sample.
    sampler = ClockSampler(local)
    sampler.start()
    sampler.wait_first()
    for _ in range(args.warmup):
        full_step()
    torch.cuda.synchronize(dev)

    import torch.distributed as dist
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    launches0 = ctx.launches
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(6)] for _ in range(args.steps)]
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for k in range(args.steps):
        full_step(ev[k])
    t1.record(stream)
    torch.cuda.synchronize(dev)
    launches = ctx.launches - launches0
    sampler.wait_next()
    clocks = sampler.stop()
    elapsed_ms = max_over_ranks(t0.elapsed_time(t1), world, dev)
    if world > 1:
        dist.barrier()
    stage_ms = {nm: 0.0 for nm in ["project_fwd", "bin", "raster_fwd", "raster_bwd", "project_bwd"]}
    for k in range(args.steps):
        e = ev[k]
        stage_ms["project_fwd"] += e[0].elapsed_time(e[1])
        stage_ms["bin"] += e[1].elapsed_time(e[2])
        stage_ms["raster_fwd"] += e[2].elapsed_time(e[3])
        stage_ms["raster_bwd"] += e[3].elapsed_time(e[4])
        stage_ms["project_bwd"] += e[4].elapsed_time(e[5])
    for k in stage_ms:
        stage_ms[k] /= args.steps
    ms_per_step = elapsed_ms / args.steps
    mpix = WIDTH * HEIGHT / 1e6
    value = mpix * world / (ms_per_step / 1e3)

    # End to end through the host-buffer C ABI (splat_renderer_submit_backward / _wait, two
    # steps in flight): the model is resident (uploaded once, as a loaded model is); every
    # step uploads its dL/dpix from pinned memory and downloads the image and the 59
    # parameter gradients into pinned memory, all inside the timed region. The synchronous
    # call (splat_renderer_render_backward, one step at a time) is timed too.
    r = G.Renderer(ctx)
    r.set_model(s["params"], 3)
    dimage_h = [torch.from_numpy(s["dimage"]).pin_memory() for _ in range(2)]
    img_h = [torch.empty(WIDTH * HEIGHT * 3, dtype=torch.float32).pin_memory() for _ in range(2)]
    grads_h = [torch.empty((n, 59), dtype=torch.float32).pin_memory() for _ in range(2)]
    e_steps = max(4, args.steps // 2)

    def pipelined(steps):
        tickets = []
        for k in range(steps):
            if k >= 2:
                r.wait(tickets[k - 2])  # host buffers of set k % 2 are free again
            tickets.append(r.submit_backward(cam, opts, bg, dimage_h[k % 2], img_h[k % 2], grads_h[k % 2]))
        for t in tickets[-2:]:
            r.wait(t)

    pipelined(max(2, args.warmup))
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    tw = time.perf_counter()
    pipelined(e_steps)
    e2e_ms = max_over_ranks((time.perf_counter() - tw) * 1e3 / e_steps, world, dev)
    sync_steps = max(3, args.steps // 10)
    tw = time.perf_counter()
    for _ in range(sync_steps):
        r.render_backward(cam, opts, bg, dimage_h[0].numpy(), img_h[0].numpy(), grads_h[0].numpy())
    sync_ms = max_over_ranks((time.perf_counter() - tw) * 1e3 / sync_steps, world, dev)
    r.close()
    e2e = {"value": round(mpix * world / (e2e_ms / 1e3), 3), "unit": UNIT,
           "h2d_bytes_per_step": int(dimage_h[0].nbytes), "d2h_bytes_per_step":
           int(img_h[0].nbytes + grads_h[0].nbytes), "ms_per_step": round(e2e_ms, 3),
           "api": "splat_renderer_submit_backward + splat_renderer_wait (2 steps in flight)",
           "synchronous_ms_per_step": round(sync_ms, 3),
           "pcie_gbs": round((dimage_h[0].nbytes + img_h[0].nbytes + grads_h[0].nbytes) / e2e_ms / 1e6, 1)}

    # Roofline per stage: max(bytes / HBM, FLOP / FP32, exp+rcp / special-function unit),
    # the HBM peak from the driver's copy measurement, FP32 and the special-function unit
    # from the microbenchmark above; the dominant kernel's goes into `roofline`.
    hbm_peak, peak_kind = measured_peaks()
    rl = stage_rooflines(stage_ms, n, entries, pairs_fwd, pairs_bwd, WIDTH * HEIGHT, hbm_peak,
                         peaks["fp32_tflops"], peaks["mufu_gops"])
    dom = max(stage_ms, key=stage_ms.get)
    d = rl[dom]
    sec = stage_ms[dom] / 1e3
    if d["bound"] == "fp32":
        achieved, peak, unit, src = d["flop"] / sec / 1e12, peaks["fp32_tflops"], "TFLOP/s", "measured (microbenchmark)"
    elif d["bound"] == "mufu":
        achieved, peak, unit, src = d["sfu"] / sec / 1e9, peaks["mufu_gops"], "Gop/s", "measured (microbenchmark)"
    else:
        achieved, peak, unit, src = d["bytes"] / sec / 1e9, hbm_peak, "GB/s", peak_kind
    # DRAM bytes per launch from one ncu capture of this workload (1M Gaussians, 1080p,
    # dram__bytes_read.sum + dram__bytes_write.sum). Other sizes have no capture.
    traffic = NCU_DRAM_BYTES_1M.get((dom,) + tuple(raster)) if n == 1_000_000 else None
    roofline = {"bound": d["bound"], "kernel": dom, "achieved": round(achieved, 3), "peak": peak, "unit": unit,
                "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": src,
                "algorithmic_bytes_per_launch": int(d["bytes"]),
                "algorithmic_flop_per_launch": int(d.get("flop", 0)),
                "algorithmic_sfu_ops_per_launch": int(d.get("sfu", 0)),
                "hbm_frac": round(d["bytes"] / sec / 1e9 / hbm_peak, 4)}
    step_roofline_ms = sum(v["roofline_ms"] for v in rl.values())
    flops = {"raster_fwd": RASTER_FWD_FLOP_PER_PAIR * pairs_fwd, "raster_bwd": RASTER_BWD_FLOP_PER_PAIR * pairs_bwd}
    compute = {k: {"pairs": p, "flop": flops[k], "ms": round(stage_ms[k], 4),
                   "tflops": round(flops[k] / (stage_ms[k] / 1e3) / 1e12, 3),
                   "ns_per_pair": round(stage_ms[k] * 1e6 / max(p, 1), 4)}
               for k, p in (("raster_fwd", pairs_fwd), ("raster_bwd", pairs_bwd))}
    hbm_stages = {
        "project_fwd": PROJ_FWD_BYTES * n, "project_bwd": PROJ_BWD_BYTES * n,
    }
    stage_hbm = {k: {"ms": round(stage_ms[k], 4), "gbs": round(v / (stage_ms[k] / 1e3) / 1e9, 1),
                     "frac": round(v / (stage_ms[k] / 1e3) / 1e9 / hbm_peak, 4)} for k, v in hbm_stages.items()}

    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded; 1M Gaussians uniform in a 10 m cube)",
        "config": workload_config(n, world),
        "raster_config": {"tile": [raster[0], raster[1]], "chunk": raster[2], "bwd_pixels_per_thread": raster[3],
                          "chosen": "autotuned" if tuning else "fixed"},
        "autotune": tuning,
        "iters_per_s": round(1e3 / ms_per_step, 3),
        "stages_ms": {k: round(v, 4) for k, v in stage_ms.items()},
        "entries": entries, "visible": visible, "sort_keys_per_s": round(entries / (stage_ms["bin"] / 1e3), 1),
        "pairs": {"fwd": pairs_fwd, "bwd": pairs_bwd},
        "e2e": e2e, "gpu_launches": int(launches), "roofline": roofline,
        "step_roofline_frac": round(step_roofline_ms / ms_per_step, 4), "step_roofline_ms": round(step_roofline_ms, 4),
        "stage_roofline": rl, "peaks": peaks, "compute": compute, "hbm_stages": stage_hbm,
        "clocks": clocks,
    }
    ctx.close()
    return line


# Plain training on the small blob scene (10k ground-truth Gaussians, 16 views at 256x256): 2,000 iterations, densification every 100
# from 500 to 1,500 (threshold 2e-4), lambda 0.2, SH degree 3 with the reference's ramp.
BLOB_TRAIN = dict(iterations=2000, densify=1, densify_from_iter=500, densify_until_iter=1500, densification_interval=100,
                densify_grad_threshold=0.0002, lambda_dssim=0.2, sh_degree=3, position_lr_max_steps=2000, seed=0)

# Plain training on the shell scene (500k ground-truth Gaussians on 40 shells, 200 views at 1297x840): the reference's defaults
# (30,000 iterations, densification 500-15,000) with at most 3,000,000 Gaussians.
SHELL_TRAIN = dict(iterations=30000, densify=1, densify_from_iter=500, densify_until_iter=15000,
                densification_interval=100, densify_grad_threshold=0.0002, lambda_dssim=0.2, sh_degree=3,
                position_lr_max_steps=30000, seed=0, max_gaussians=3_000_000)


# Batched mixed-precision training on the same scene with mixed view sizes: 8 views of mixed sizes per
# step, BF16 render copy, f64 conic re-solve, graph replay; as many views as the plain
# run (3,750 steps of 8) with the plain schedule in views (every step-count divided by 8).
BATCHED_TRAIN = dict(iterations=3750, densify=1, densify_from_iter=63, densify_until_iter=1875, densification_interval=13,
                opacity_reset_interval=375, densify_grad_threshold=0.0002, lambda_dssim=0.2, sh_degree=3,
                sh_degree_interval=125, position_lr_max_steps=3750, seed=0, max_gaussians=3_000_000,
                batch_views=8, bf16_storage=1, fp64_conic=1, autotune=1)


def gt_views_gpu(ctx, s):
    """Target views: the ground truth rendered by the device renderer, as 8-bit images."""
    from splatrs_b200 import gpu as G
    from splatrs_b200 import scenes
    from splatrs_b200._lib import Camera, ProjOpts
    r = G.Renderer(ctx)
    r.set_model(s["gt"], 3)
    views = [(cam, scenes.to_rgb8(r.render(Camera.from_record(cam), ProjOpts.make(sh_degree=3), (0, 0, 0))))
             for cam in s["cams"]]
    r.close()
    return views


# Learned densification's labels and policy: a kept Gaussian whose descendants blended
# less than 10 pixel-equivalents over a densification window (13 steps of 8 views) is
# labelled prune, and applying prunes at a prune probability of 0.95.
LEARN_SETTINGS = dict(learn_contribution=10.0, learn_prune_confidence=0.95)


def run_learned_densify(local, learn_iters, learn=None, plain=True):
    """Learned densification on the shell scene with mixed view sizes, BF16 storage and f64 conics: the network
    learns online from plain runs on scene seeds 2-5 (the densification window of each),
    then plain and learned densification train scene seed 6 for the same number of steps."""
    learn_cfg = dict(LEARN_SETTINGS if learn is None else learn)
    import torch
    from splatrs_b200 import gpu as G
    from splatrs_b200 import scenes
    ctx = G.Context(local, torch.cuda.current_stream(local))

    def setup(seed):
        s = scenes.shell_scene_mixed_sizes(seed_gt=seed, seed_init=seed + 100)
        views = gt_views_gpu(ctx, s)
        ip = G.init_from_points(ctx, s["init_points"], s["init_rgb"])
        n0 = len(s["init_points"])
        init = G.planes_to_params(ctx, ip, n0, n0).cpu().numpy()
        return init, views, scenes.scene_extent(s["cams"])

    theta, learn_log = None, []
    for seed in (2, 3, 4, 5):
        init, views, ext = setup(seed)
        t = G.Trainer(ctx, init, ext, views, **dict(BATCHED_TRAIN, learned_densify=1, **learn_cfg))
        if theta is not None:
            t.set_mlp(theta)
        tw = time.perf_counter()
        t.run(learn_iters)
        torch.cuda.synchronize(local)
        st = t.mlp_stats()
        theta = t.get_mlp()
        learn_log.append({"seed": seed, "steps": learn_iters, "wall_s": round(time.perf_counter() - tw, 2),
                      "densifications": st["events"], "records": st["records"],
                      "labels_keep_densify_prune": [st["label_keep"], st["label_densify"], st["label_prune"]],
                      "heldout_accuracy_network": round(st["heldout_net"] / max(st["heldout_records"], 1), 4),
                      "heldout_accuracy_rule": round(st["heldout_rule"] / max(st["heldout_records"], 1), 4)})
        t.close()
    init, views, ext = setup(6)
    ev = {}
    for name, mode in ((("plain", 0),) if plain else ()) + (("learned", 2),):
        t = G.Trainer(ctx, init, ext, views, **dict(BATCHED_TRAIN, learned_densify=mode, **(learn_cfg if mode else {})))
        if mode == 2:
            t.set_mlp(theta)
        torch.cuda.synchronize(local)
        tw = time.perf_counter()
        t.run(BATCHED_TRAIN["iterations"])
        torch.cuda.synchronize(local)
        wall = time.perf_counter() - tw
        sc = t.evaluate()  # splat_trainer_evaluate: every view scored on the device
        ev[name] = {"steps": BATCHED_TRAIN["iterations"], "wall_s": round(wall, 3), "psnr_train_views": round(sc["psnr"], 2),
                    "ssim_train_views": round(sc["ssim"], 4), "gaussians": t.count}
        t.close()
    ctx.close()
    return {"labels": learn_cfg, "learn": learn_log, "seed6": ev}


def target_config(batch, coarse_frac=2.0 / 3.0, views_total=30000, threshold=0.0002):
    """The batched, coarse-to-fine trainer's schedule: the plain trainer's 30,000-view schedule
    in steps of `batch` views (every step count divided by the batch), learning rates scaled
    by sqrt(batch) (Adam's step does not grow with the summed gradient), and the first
    `coarse_frac` of the steps on the views box-filtered by 2."""
    it = views_total // batch
    sc = math.sqrt(batch)
    return dict(iterations=it, densify=1, densify_from_iter=500 // batch, densify_until_iter=15000 // batch,
                densification_interval=max(1, 100 // batch), opacity_reset_interval=3000 // batch,
                densify_grad_threshold=threshold, lambda_dssim=0.2, sh_degree=3,
                sh_degree_interval=max(1, 1000 // batch), position_lr_max_steps=it, seed=0, max_gaussians=3_000_000,
                batch_views=batch, position_lr_init=0.00016 * sc, position_lr_final=0.0000016 * sc,
                feature_lr=0.0025 * sc, opacity_lr=0.025 * sc, scaling_lr=0.005 * sc, rotation_lr=0.001 * sc,
                coarse_until=int(it * coarse_frac), coarse_factor=2)


# The training target's trainer: batches of TARGET_BATCH views, coarse-to-fine, learned
# densification (learned on scene seeds 2-5, applied on seed 6), graph-replayed.
TARGET_BATCH = 2
TARGET_THRESHOLD = 0.0002
# The network's contribution threshold counts pixels of the views it trains on, which are
# the half-resolution ones while densification runs: 9.5 there is about 38 full-resolution
# pixel-equivalents. Swept on this protocol (scene seed 6, two or three runs each): 2.5 ->
# 0.92x the plain count at +0.7 dB; 4 -> 0.88x, +0.6 dB; 6 -> 0.79-0.86x, +0.2-0.5 dB;
# 8 -> 0.75-0.81x, +0.1-0.4 dB. With the paired compositing backward the network learns
# from slightly different records: 9 -> 0.79-0.80x, +0.28/+0.36 dB; 9.5 -> 0.762-0.764x,
# +0.07 to +0.18 dB (four runs, two networks); 10 -> 0.72-0.76x, -0.18 to +0.12 dB (two
# networks); 11 -> 0.72x, -0.12/-0.08 dB.
TARGET_LEARN = dict(learn_contribution=9.5, learn_prune_confidence=0.95)
TARGET_RUNS = 2  # the target trainer runs this many times with the one learned network


def run_train_target(local):
    """The training target on the clustered 500k-Gaussian scene (seed 6), all 200 views at
    1297x840: the plain one-view trainer (30,000 iterations, the reference's schedule)
    against the batched, graph-replayed, coarse-to-fine trainer with learned densification
    (the same 30,000 views), whose network first learns on four other scenes (seeds 2-5) with
    the same schedule up to the end of densification. Reports each run's wall time, PSNR
    over the 200 views at full resolution and Gaussian count, and the three ratios the
    target sets bars on: PSNR within 0.1 dB of plain's, at least 1.5x less wall time, at
    most 0.8x the Gaussians."""
    import torch
    from splatrs_b200 import gpu as G
    from splatrs_b200 import scenes
    ctx = G.Context(local, torch.cuda.current_stream(local))

    def setup(seed):
        sc = scenes.shell_scene(seed_gt=seed, seed_init=seed + 100)
        views = gt_views_gpu(ctx, sc)
        ip = G.init_from_points(ctx, sc["init_points"], sc["init_rgb"])
        n0 = len(sc["init_points"])
        init = G.planes_to_params(ctx, ip, n0, n0).cpu().numpy()
        return init, views, scenes.scene_extent(sc["cams"])

    def train(init, views, ext, cfg, theta=None, iterations=None):
        t = G.Trainer(ctx, init, ext, views, **cfg)
        if theta is not None:
            t.set_mlp(theta)
        torch.cuda.synchronize(local)
        tw = time.perf_counter()
        t.run(iterations or cfg["iterations"])
        torch.cuda.synchronize(local)
        wall = time.perf_counter() - tw
        return t, wall

    tcfg = target_config(TARGET_BATCH, threshold=TARGET_THRESHOLD)
    theta, learn_log = None, []
    for seed in (2, 3, 4, 5):
        init, views, ext = setup(seed)
        steps = tcfg["densify_until_iter"] + 2 * tcfg["densification_interval"]
        t, wall = train(init, views, ext, dict(tcfg, learned_densify=1, **TARGET_LEARN), theta, steps)
        st = t.mlp_stats()
        theta = t.get_mlp()
        learn_log.append({"seed": seed, "steps": steps, "wall_s": round(wall, 2), "records": st["records"],
                          "heldout_accuracy_network": round(st["heldout_net"] / max(st["heldout_records"], 1), 4),
                          "heldout_accuracy_rule": round(st["heldout_rule"] / max(st["heldout_records"], 1), 4)})
        t.close()
        del views
    init, views, ext = setup(6)

    def scored(cfg, th):
        t, wall = train(init, views, ext, cfg, th)
        ev = t.evaluate()
        r = {"views_per_step": int(cfg.get("batch_views", 1) or 1), "steps": cfg["iterations"],
             "wall_s": round(wall, 2), "psnr": round(ev["psnr"], 3), "ssim": round(ev["ssim"], 4), "gaussians": t.count}
        t.close()
        return r

    p = scored(SHELL_TRAIN, None)
    runs = [scored(dict(tcfg, learned_densify=2, **TARGET_LEARN), theta) for _ in range(TARGET_RUNS)]
    ctx.close()

    def ratios(q):
        r = {"psnr_diff_db": round(q["psnr"] - p["psnr"], 3), "wall_time_ratio": round(p["wall_s"] / q["wall_s"], 3),
             "gaussian_ratio": round(q["gaussians"] / max(p["gaussians"], 1), 3)}
        r["bars_met"] = {"psnr_within_0.1db_or_above": r["psnr_diff_db"] >= -0.1,
                         "wall_time_ratio_at_least_1.5": r["wall_time_ratio"] >= 1.5,
                         "gaussian_ratio_at_most_0.8": r["gaussian_ratio"] <= 0.8}
        return r

    mean = {k: round(float(np.mean([r[k] for r in runs])), 3) for k in ("wall_s", "psnr", "ssim", "gaussians")}
    out = {"scene": "500k Gaussians on 40 shells, seed 6; 200 views at 1297x840",
           "plain": p, "target_runs": [dict(r, **ratios(r)) for r in runs], "target_mean": dict(mean, **ratios(mean)),
           "learn": learn_log,
           "target_settings": {"batch_views": TARGET_BATCH, "coarse": "first 2/3 of the steps at half resolution",
                               "lr_scale": round(math.sqrt(TARGET_BATCH), 3), "densify_grad_threshold": TARGET_THRESHOLD,
                               "learned_densify": "apply", "runs_with_one_network": TARGET_RUNS, **TARGET_LEARN}}
    return out


def run_train_gpu(local, s, cfg, iterations, snapshots=()):
    """A plain training run on the device trainer: wall time, iterations/s, PSNR over the
    training views, final Gaussian count. Targets and initial model are built on the
    device before the clock starts. `snapshots`: iteration numbers at which the model is
    copied out (the run pauses there; the copy is outside the clock), returned with the
    result as out["snapshots"] = [(iteration, model)], the initial model first."""
    import torch
    from splatrs_b200 import gpu as G
    from splatrs_b200 import scenes
    ctx = G.Context(local, torch.cuda.current_stream(local))
    views = gt_views_gpu(ctx, s)
    init_planes = G.init_from_points(ctx, s["init_points"], s["init_rgb"])
    n0 = len(s["init_points"])
    init = G.planes_to_params(ctx, init_planes, n0, n0).cpu().numpy()
    del init_planes
    extent = scenes.scene_extent(s["cams"])
    t = G.Trainer(ctx, init, extent, views, **cfg)
    snaps = [(0, init)] if snapshots else []
    wall, done = 0.0, 0
    for stop in sorted(set(int(x) for x in snapshots if 0 < x < iterations)) + [iterations]:
        torch.cuda.synchronize(local)
        tw = time.perf_counter()
        t.run(stop - done)  # splat_trainer_run: the segment in one call, queued ahead of the device
        torch.cuda.synchronize(local)
        wall += time.perf_counter() - tw
        done = stop
        if snapshots:
            snaps.append((stop, t.model()))
    ev = t.evaluate()  # splat_trainer_evaluate: every view scored on the device
    bv = max(1, int(cfg.get("batch_views", 1)))
    out = {"iterations": iterations, "wall_s": round(wall, 3), "iters_per_s": round(iterations / wall, 1),
           "views_per_s": round(iterations * bv / wall, 1), "psnr_train_views": round(ev["psnr"], 2),
           "ssim_train_views": round(ev["ssim"], 4), "gaussians": t.count}
    if cfg.get("autotune"):
        tu = t.tuning()
        out["autotune"] = {"tunes": tu["tunes"], "picked": list(tu["picked"]),
                           "ms_per_pass": {f"{a}x{b}x{c}/{d}": round(v, 4) for (a, b, c, d), v in tu["ms"].items()}}
    if snapshots:
        out["snapshots"] = snaps
    t.close()
    ctx.close()
    return out, init, views, extent


def run_train_cpu_states(snaps, views, extent, cfg, iters, total_iters):
    """CPU oracle time per iteration at several model states of a GPU run (the model copied
    out at those iterations; fresh Adam moments, no densification, the SH degree ramped to
    its final value over 3 untimed iterations, then `iters` timed ones), and the run's CPU
    time extrapolated from them by the trapezoid rule over the iterations between states."""
    from oracle import oracle as O
    ccfg = {k: v for k, v in cfg.items() if k not in ("max_gaussians", "autotune")}
    ccfg.update(densify=0, sh_degree_interval=1)
    rows = []
    for it, model in snaps:
        ot = O.Trainer(model, extent, views, **ccfg)
        for _ in range(3):
            ot.step()
        tw = time.perf_counter()
        for _ in range(iters):
            ot.step()
        rows.append({"iteration": it, "gaussians": int(model.shape[0]),
                     "s_per_iter": round((time.perf_counter() - tw) / iters, 4)})
        del ot
    est = 0.0
    for a, b in zip(rows[:-1], rows[1:]):
        est += 0.5 * (a["s_per_iter"] + b["s_per_iter"]) * (b["iteration"] - a["iteration"])
    return {"states": rows, "extrapolated_s": round(est, 1), "iterations": total_iters,
            "extrapolated_iters_per_s": round(total_iters / est, 4) if est > 0 else None, "cores": O.threads(),
            "kind": "port",
            "sample": (f"{iters} timed iterations (after 3 untimed) at each model state of the GPU run; the "
                       f"{total_iters}-iteration CPU time is EXTRAPOLATED by the trapezoid rule between states")}


def run_blob_seeds(local, seeds=(0, 1, 2, 3, 4)):
    """The small blob scene trained with the default backward (float atomics: sums in no
    fixed order) and with the deterministic one (the reference's reduction; bit-identical to
    the oracle trainer with correctly rounded exp/log, which the GPU tests check), for
    trainer seeds 0-4 (view order and split draws): the PSNR gap atomic - deterministic per
    seed, its mean and spread, and both modes' iterations per second."""
    import torch
    from splatrs_b200 import gpu as G
    from splatrs_b200 import scenes
    ctx = G.Context(local, torch.cuda.current_stream(local))
    s = scenes.blob_scene()
    views = gt_views_gpu(ctx, s)
    ip = G.init_from_points(ctx, s["init_points"], s["init_rgb"])
    n0 = len(s["init_points"])
    init = G.planes_to_params(ctx, ip, n0, n0).cpu().numpy()
    del ip
    extent = scenes.scene_extent(s["cams"])
    rows = []
    for seed in seeds:
        row = {"seed": seed}
        for name, det in (("atomic", 0), ("deterministic", 1)):
            t = G.Trainer(ctx, init, extent, views, **dict(BLOB_TRAIN, seed=seed, deterministic=det))
            torch.cuda.synchronize(local)
            tw = time.perf_counter()
            t.run(BLOB_TRAIN["iterations"])
            torch.cuda.synchronize(local)
            wall = time.perf_counter() - tw
            row[name] = {"psnr": round(t.evaluate()["psnr"], 3), "gaussians": t.count,
                         "iters_per_s": round(BLOB_TRAIN["iterations"] / wall, 1)}
            t.close()
        row["gap_db"] = round(row["atomic"]["psnr"] - row["deterministic"]["psnr"], 3)
        rows.append(row)
    ctx.close()
    gaps = np.array([r["gap_db"] for r in rows])
    return {"seeds": rows, "mean_gap_db": round(float(gaps.mean()), 3), "std_gap_db": round(float(gaps.std(ddof=1)), 3),
            "max_abs_gap_db": round(float(np.abs(gaps).max()), 3),
            "note": "deterministic = the reference's reduction order, bit-identical to the correctly rounded "
                    "oracle trainer (tests/test_gpu_deterministic.py); atomic = the default float-atomic backward"}


def run_train_cpu(init, views, extent, cfg, iterations):
    """The same run on the CPU oracle trainer (all host threads), for `iterations` steps."""
    from oracle import oracle as O
    from splatrs_b200 import scenes
    ot = O.Trainer(init, extent, views, **{k: v for k, v in cfg.items() if k not in ("max_gaussians", "autotune")})
    tw = time.perf_counter()
    for _ in range(iterations):
        ot.step()
    wall = time.perf_counter() - tw
    out = {"iterations": iterations, "wall_s": round(wall, 3), "iters_per_s": round(iterations / wall, 3),
           "gaussians": ot.count, "cores": O.threads(), "kind": "port"}
    if iterations == cfg["iterations"]:
        out["psnr_train_views"] = round(float(np.mean([scenes.psnr(ot.render(cam), rgb) for cam, rgb in views])), 2)
    return out


def cpu_reference_steps(args, steps, warmup=1):
    """The CPU oracle (the reference's hot path restated in C++, all host threads) on the
    same workload: `steps` full forward+backward passes of the 1920x1080 view. Returns the
    mean seconds per step, the threads used and a per-stage breakdown (as the reference's
    examples/profile.rs reports it) with the compositing cost in ns per pair per core, over
    the pairs that pass the alpha threshold: the unit of the reference's published figures
    (README.md:153: ~15 ns forward, ~25 ns backward)."""
    from oracle import oracle as O
    from splatrs_b200 import scenes
    s = scenes.render_benchmark_scene(n=args.n)
    p, cam, dimage = s["params"], s["cam"], s["dimage"]
    bg = np.zeros(3, np.float32)
    names = ("project", "bin", "raster_fwd", "raster_bwd", "project_bwd")
    acc = dict.fromkeys(names, 0.0)
    passed = [0, 0]

    def one(record):
        t = [time.perf_counter()]
        projs = O.project_all(p, cam, sh_degree=3)
        t.append(time.perf_counter())
        b = O.bin(projs, WIDTH, HEIGHT)
        t.append(time.perf_counter())
        img, ft, nc, _ = O.rasterize_forward(projs, b, WIDTH, HEIGHT, bg)
        t.append(time.perf_counter())
        g, a, _ = O.rasterize_backward(projs, b, WIDTH, HEIGHT, bg, ft, nc, dimage)
        t.append(time.perf_counter())
        O.project_backward_all(p, cam, g, sh_degree=3)
        t.append(time.perf_counter())
        if record:
            for k, nm in enumerate(names):
                acc[nm] += t[k + 1] - t[k]
            passed[:] = O.last_passed_pairs()

    for _ in range(max(1, warmup)):
        one(False)  # warm caches and thread pool
    t0 = time.perf_counter()
    for _ in range(steps):
        one(True)
    dt = (time.perf_counter() - t0) / steps
    cores = O.threads()
    ms = {nm: round(acc[nm] / steps * 1e3, 2) for nm in names}
    detail = {"stages_ms": ms, "passed_pairs": {"forward": passed[0], "backward": passed[1]},
              "ns_per_pair_core": {"forward": round(ms["raster_fwd"] * 1e6 * cores / max(passed[0], 1), 2),
                                   "backward": round(ms["raster_bwd"] * 1e6 * cores / max(passed[1], 1), 2),
                                   "reference_published": {"forward": 15, "backward": 25}}}
    return dt, cores, detail


ADAM_BYTES = 4 * 240 + 3 * 240            # params, grads, m, v read; params, m, v written (60 floats padded)
PROJ_BWD_ADAM_BYTES = 240 + 64 + 48 + 2 * 240 + 3 * 240  # + record and screen gradients; no gradient round trip
LOSS_BYTES_PER_PIXEL = 12 + 3 + 12        # prediction read, u8 target read, gradient written
LOSS_FLOP_PER_PIXEL = 1056                # five blurs forward, three back, SSIM and its partials, L1


def run_stages(local, reps=20):
    """The HBM- or FP32-bound stages outside the render step, CUDA-event timed on their own
    (inputs above L2): the fused SSIM + L1 loss forward and backward on one 1297x840 view,
    Adam over 1M Gaussians, and the projection backward fused with Adam over 1M Gaussians
    (the trainer's optimiser step)."""
    import torch
    from splatrs_b200 import gpu as G
    from splatrs_b200 import scenes
    from splatrs_b200._lib import Camera, LearningRates, ProjOpts
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    ctx = G.Context(local, stream)
    hbm, kind = measured_peaks()
    fp32_peak = max(ctx.peak("fp32")["ops_per_s"] for _ in range(3)) / 1e12  # measured, TFLOP/s

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / reps

    out = {"peak_hbm_gbs": hbm, "peak_source": kind, "fp32_tflops_measured": round(fp32_peak, 1)}
    w, h = 1297, 840
    rng = np.random.default_rng(3)
    pred = torch.from_numpy(rng.uniform(0, 1, w * h * 3).astype(np.float32)).to(dev)
    tgt = torch.from_numpy(rng.integers(0, 256, w * h * 3).astype(np.uint8)).to(dev)
    grad = torch.empty_like(pred)
    lo = torch.empty(3, dtype=torch.float32, device=dev)
    ms = timed(lambda: G.check(ctx.lib.splat_loss_fwd_bwd(ctx.h, G._ptr(pred), G._ptr(tgt), 1, w, h, 0.2,
                                                          G._ptr(grad), G._ptr(lo)), ctx.h))
    px = w * h
    out["ssim_l1_fwd_bwd"] = {"pixels": px, "ms": round(ms, 4), "bytes_per_pixel": LOSS_BYTES_PER_PIXEL,
                              "gbs": round(LOSS_BYTES_PER_PIXEL * px / ms / 1e6, 1),
                              "hbm_frac": round(LOSS_BYTES_PER_PIXEL * px / ms / 1e6 / hbm, 4),
                              "flop_per_pixel": LOSS_FLOP_PER_PIXEL,
                              "tflops": round(LOSS_FLOP_PER_PIXEL * px / ms / 1e9, 2),
                              "fp32_frac": round(LOSS_FLOP_PER_PIXEL * px / ms / 1e9 / fp32_peak, 4)}
    del pred, tgt, grad
    n = 1_000_000
    sc = scenes.render_benchmark_scene(n=n)
    planes = G.params_to_planes(ctx, torch.from_numpy(sc["params"]).to(dev))
    grads = torch.randn_like(planes) * 1e-3
    m, v = torch.zeros_like(planes), torch.zeros_like(planes)
    lr = LearningRates(mean=1.6e-4, log_scale=0.005, quat=0.001, opacity=0.025, sh_dc=0.0025, sh_rest=0.000125)
    step = [0]

    def adam():
        step[0] += 1
        G.adam_step(ctx, planes, grads, m, v, n, n, step[0], lr)

    ms = timed(adam)
    out["adam"] = {"gaussians": n, "ms": round(ms, 4), "bytes_per_gaussian": ADAM_BYTES,
                   "gbs": round(ADAM_BYTES * n / ms / 1e6, 1), "hbm_frac": round(ADAM_BYTES * n / ms / 1e6 / hbm, 4)}
    cam, opts = Camera.from_record(sc["cam"]), ProjOpts.make(sh_degree=3)
    proj = G.project_all(ctx, planes, n, n, cam, opts)
    pgrad = torch.randn((3, n, 4), dtype=torch.float32, device=dev) * 1e-3

    def pba():
        step[0] += 1
        G.project_backward_adam(ctx, planes, m, v, n, n, cam, opts, proj, pgrad, step[0], lr)

    ms = timed(pba)
    out["project_bwd_adam"] = {"gaussians": n, "ms": round(ms, 4), "bytes_per_gaussian": PROJ_BWD_ADAM_BYTES,
                               "gbs": round(PROJ_BWD_ADAM_BYTES * n / ms / 1e6, 1),
                               "hbm_frac": round(PROJ_BWD_ADAM_BYTES * n / ms / 1e6 / hbm, 4)}
    ctx.close()
    return out


def run_mlp(local, rows, reps=20):
    """The learned-densification network's forward on `rows` feature rows already on the
    device: the tcgen05 kernel (what the trainer runs) and the mma.sync kernel, CUDA-event
    timed per call on the launching stream (each call synchronises once for its timeout
    check, so the figure includes one host round trip)."""
    import torch
    from oracle import mlp as M
    from splatrs_b200 import gpu as G
    dev = torch.device("cuda", local)
    ctx = G.Context(local, torch.cuda.current_stream(local))
    rng = np.random.default_rng(1)
    x = torch.from_numpy(rng.normal(0, 1, (rows, 16)).astype(np.float32)).to(dev)
    th = torch.from_numpy(M.init_params(1).astype(np.float32)).to(dev)
    out = {"rows": rows, "flop_per_row": 2 * (16 * 64 + 64 * 64 + 64 * 3), "bytes_per_row": 16 * 4 + 3 * 4}
    stream = torch.cuda.current_stream(dev)
    for name, tc in (("tcgen05", True), ("mma_sync", False)):
        for _ in range(3):
            G.mlp_forward(ctx, x, th, tcgen05=tc)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            G.mlp_forward(ctx, x, th, tcgen05=tc)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / reps
        out[name] = {"ms": round(ms, 4), "tflops": round(out["flop_per_row"] * rows / ms / 1e9, 2),
                     "gbs": round(out["bytes_per_row"] * rows / ms / 1e6, 1)}
    # The gradient over the same rows (labels and weights drawn alike): forward and backward,
    # 3 x the forward's multiply-adds per row.
    yl = torch.from_numpy(rng.integers(0, 3, rows).astype(np.int32)).to(dev)
    wl = torch.from_numpy(rng.uniform(0.2, 2.0, rows).astype(np.float32)).to(dev)
    grad = torch.zeros(int(M.NUM_PARAMS), dtype=torch.float32, device=dev)
    out["grad_flop_per_row"] = 3 * out["flop_per_row"]
    for name, tc in (("grad_tcgen05", True), ("grad_mma_sync", False)):
        fn = ctx.lib.splat_mlp_grad_tc if tc else ctx.lib.splat_mlp_grad
        call = lambda: G.check(fn(ctx.h, G._ptr(x), G._ptr(yl), G._ptr(wl), rows, 1.0 / rows, G._ptr(th),
                                  G._ptr(grad)), ctx.h)
        for _ in range(3):
            call()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            call()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / reps
        out[name] = {"ms": round(ms, 4), "tflops": round(out["grad_flop_per_row"] * rows / ms / 1e9, 2)}
    ctx.close()
    return out


def run_profile_stages(local):
    """The HBM-bound stages for an ncu capture, each run twice (skip the first of each):
    projection forward, projection backward and Adam over the render benchmark's 1M
    Gaussians, and the fused SSIM + L1 loss forward and backward on one 1297x840 view
    (u8 target). About 1.5 GB on the device."""
    import torch
    from splatrs_b200 import gpu as G
    from splatrs_b200 import scenes
    from splatrs_b200._lib import Camera, LearningRates, ProjOpts
    dev = torch.device("cuda", local)
    ctx = G.Context(local, torch.cuda.current_stream(dev))
    n = 1_000_000
    sc = scenes.render_benchmark_scene(n=n)
    planes = G.params_to_planes(ctx, torch.from_numpy(sc["params"]).to(dev))
    cam, opts = Camera.from_record(sc["cam"]), ProjOpts.make(sh_degree=3)
    pgrad = torch.randn((3, n, 4), dtype=torch.float32, device=dev) * 1e-3
    grads = torch.randn_like(planes) * 1e-3
    m, v = torch.zeros_like(planes), torch.zeros_like(planes)
    lr = LearningRates(mean=1.6e-4, log_scale=0.005, quat=0.001, opacity=0.025, sh_dc=0.0025, sh_rest=0.000125)
    w, h = 1297, 840
    rng = np.random.default_rng(3)
    pred = torch.from_numpy(rng.uniform(0, 1, w * h * 3).astype(np.float32)).to(dev)
    tgt = torch.from_numpy(rng.integers(0, 256, w * h * 3).astype(np.uint8)).to(dev)
    lgrad = torch.empty_like(pred)
    lo = torch.empty(3, dtype=torch.float32, device=dev)
    for rep in range(2):
        proj = G.project_all(ctx, planes, n, n, cam, opts)
        G.project_backward_all(ctx, planes, n, n, cam, opts, proj, pgrad)
        G.adam_step(ctx, planes, grads, m, v, n, n, rep + 1, lr)
        G.check(ctx.lib.splat_loss_fwd_bwd(ctx.h, G._ptr(pred), G._ptr(tgt), 1, w, h, 0.2, G._ptr(lgrad), G._ptr(lo)),
                ctx.h)
    torch.cuda.synchronize(dev)
    ctx.close()
    return {"profile_stages": {"gaussians": n, "loss_view": [w, h], "reps": 2}}


def run_profile_blobs(local):
    """Config-0 training for an ncu launch list: the blob scene, 300 plain iterations
    (densification from 100 every 100, SH degree ramped every 50). Prints how many kernel
    launches come before the last 100 iterations and how many those take."""
    import torch
    from splatrs_b200 import gpu as G
    from splatrs_b200 import scenes
    s = scenes.blob_scene()
    ctx = G.Context(local, torch.cuda.current_stream(local))
    views = gt_views_gpu(ctx, s)
    ip = G.init_from_points(ctx, s["init_points"], s["init_rgb"])
    n0 = len(s["init_points"])
    init = G.planes_to_params(ctx, ip, n0, n0).cpu().numpy()
    cfg = dict(BLOB_TRAIN, iterations=300, densify_from_iter=100, densify_until_iter=199, densification_interval=100,
               sh_degree_interval=50, position_lr_max_steps=300)
    t = G.Trainer(ctx, init, scenes.scene_extent(s["cams"]), views, **cfg)
    t.run(200)
    torch.cuda.synchronize(local)
    before = ctx.launches
    t.run(100)
    torch.cuda.synchronize(local)
    out = {"profile_blobs": {"launches_before_last_100": before, "launches_last_100": ctx.launches - before,
                             "gaussians": t.count}}
    t.close()
    ctx.close()
    return out


def run_profile_train(local):
    """Config-2 training for an ncu launch list: the scene's first 20 cameras, 300 plain
    iterations (densification from 100 every 50). Prints how many kernel launches come
    before the last 100 iterations (skip that many) and how many those take."""
    import torch
    from splatrs_b200 import gpu as G
    from splatrs_b200 import scenes
    s = scenes.shell_scene()
    s["cams"] = s["cams"][:20]
    ctx = G.Context(local, torch.cuda.current_stream(local))
    views = gt_views_gpu(ctx, s)
    init_planes = G.init_from_points(ctx, s["init_points"], s["init_rgb"])
    n0 = len(s["init_points"])
    init = G.planes_to_params(ctx, init_planes, n0, n0).cpu().numpy()
    cfg = dict(SHELL_TRAIN, iterations=300, densify_from_iter=100, densify_until_iter=250, densification_interval=50,
               position_lr_max_steps=300)
    t = G.Trainer(ctx, init, scenes.scene_extent(s["cams"]), views, **cfg)
    t.run(200)
    torch.cuda.synchronize(local)
    before = ctx.launches
    t.run(100)
    torch.cuda.synchronize(local)
    out = {"profile_train": {"launches_before_last_100": before, "launches_last_100": ctx.launches - before,
                             "gaussians": t.count}}
    t.close()
    ctx.close()
    return out


def main():
    args = parse()
    if args.profile_train:
        print(json.dumps(run_profile_train(0)), flush=True)
        return
    if args.profile_blobs:
        print(json.dumps(run_profile_blobs(0)), flush=True)
        return
    if args.profile_mlp:
        print(json.dumps({"mlp": run_mlp(0, args.mlp_rows, reps=3)}), flush=True)
        return
    if args.profile_stages:
        print(json.dumps(run_profile_stages(0)), flush=True)
        return
    rank, world, local = dist_info()
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        gpu = torch.cuda.is_available()
        if gpu:
            torch.cuda.set_device(local)
        # NCCL on the GPU box; gloo where there is no GPU (the CPU reference arm).
        dist.init_process_group("nccl" if gpu else "gloo", timeout=timedelta(seconds=300))
    if args.profile_small:
        args.n = 200_000
        args.steps = 1
        args.warmup = 1
        args.no_cpu_baseline = True

    if args.impl == "reference":
        if rank == 0:
            # Each CPU step takes about 0.6 s on 16 host threads: up to 200 steps and 20
            # warm-up steps keep the run within a few minutes; more are capped (and said so).
            steps, warmup = max(1, min(args.steps, REF_MAX_STEPS)), max(1, min(args.warmup, REF_MAX_WARMUP))
            dt, cores, detail = cpu_reference_steps(args, steps, warmup)
            v = WIDTH * HEIGHT / 1e6 / dt
            line = {"impl": "reference", "metric": METRIC, "value": round(v, 4), "unit": UNIT, "n_gpus": world,
                    "steps": steps, "warmup": warmup, "ms_per_step": round(dt * 1e3, 2), "higher_is_better": True,
                    "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                    "data": "synthetic (seeded; 1M Gaussians uniform in a 10 m cube)",
                    "config": workload_config(args.n, world),
                    "cpu_baseline": {"value": round(v, 4), "unit": UNIT, "cores": cores, "kind": "port",
                                     "sample": f"{steps} full fwd+bwd steps of the workload", **detail},
                    "e2e": {"value": round(v, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
            if steps != args.steps or warmup != args.warmup:
                line["capped"] = (f"--steps {args.steps} --warmup {args.warmup} capped to {steps}/{warmup} "
                                  f"(about 0.6 s per CPU step)")
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
        return

    line = run_ours(args, rank, world, local)

    def leg(name, fn):
        """Runs one optional leg; a failure is recorded in the line instead of losing it."""
        try:
            return fn()
        except Exception as e:  # noqa: BLE001 - the headline line must survive any leg
            import traceback
            traceback.print_exc()
            line.setdefault("leg_errors", {})[name] = f"{type(e).__name__}: {e}"
            return None

    if not args.profile_small:
        line["mlp"] = leg("mlp", lambda: run_mlp(local, args.mlp_rows))
        line["stages"] = leg("stages", lambda: run_stages(local))
    blobs = None
    train_legs = not args.profile_small and not args.no_train and world == 1
    if train_legs:
        from splatrs_b200 import scenes

        def blob_leg():
            gpu_blobs, init, views, extent = run_train_gpu(local, scenes.blob_scene(), BLOB_TRAIN,
                                                           BLOB_TRAIN["iterations"])
            return {"gpu": gpu_blobs}, (init, views, extent)
        r = leg("train_blobs", blob_leg)
        if r is not None:
            line["train_blobs"], blobs = r
            line["train_blobs"]["atomic_vs_deterministic"] = leg("atomic_vs_deterministic",
                                                                 lambda: run_blob_seeds(local))
    if train_legs and not args.no_train_shells:
        from splatrs_b200 import scenes

        def shells_leg():
            iters = args.train_shells_iters or SHELL_TRAIN["iterations"]
            marks = [m for m in (7000, 15000) if m < iters]
            gpu_shells, init2, views2, extent2 = run_train_gpu(local, scenes.shell_scene(), SHELL_TRAIN, iters, marks)
            snaps = gpu_shells.pop("snapshots", [])
            out = {"gpu": gpu_shells}
            if rank == 0 and args.shells_cpu_iters > 0 and not args.no_cpu_baseline:
                cpu = run_train_cpu_states(snaps, views2, extent2, SHELL_TRAIN, args.shells_cpu_iters, iters)
                out["cpu"] = cpu
                if cpu["extrapolated_s"]:
                    out["gpu_over_cpu_extrapolated"] = round(cpu["extrapolated_s"] / gpu_shells["wall_s"], 1)
            return out
        line["train_shells"] = leg("train_shells", shells_leg)
    if train_legs and args.train_batched:
        from splatrs_b200 import scenes

        def batched_leg():
            iters = args.train_batched_iters or BATCHED_TRAIN["iterations"]
            gpu_batched, _, _, _ = run_train_gpu(local, scenes.shell_scene_mixed_sizes(), BATCHED_TRAIN, iters)
            return {"gpu": gpu_batched, "views_per_step": BATCHED_TRAIN["batch_views"],
                    "sizes": "uniform over 640x480, 1024x768, 1297x840, 1600x1200 per view"}
        line["train_batched"] = leg("train_batched", batched_leg)
    if train_legs and args.train_learned:
        line["train_learned"] = leg("train_learned", lambda: run_learned_densify(local, args.learn_iters))
    if train_legs and not args.no_train_target:
        line["train_target"] = leg("train_target", lambda: run_train_target(local))
    if rank == 0:
        if blobs is not None and not args.no_cpu_baseline and world == 1:
            line["train_blobs"]["cpu"] = leg("train_blobs_cpu",
                                             lambda: run_train_cpu(*blobs, BLOB_TRAIN, BLOB_TRAIN["iterations"]))
        if not args.no_cpu_baseline and world == 1:
            dt, cores, detail = cpu_reference_steps(args, args.cpu_steps)
            line["cpu_baseline"] = {"value": round(WIDTH * HEIGHT / 1e6 / dt, 4), "unit": UNIT, "cores": cores,
                                    "kind": "port", "sample": f"{args.cpu_steps} full fwd+bwd steps of the workload",
                                    **detail}
        elif world > 1:
            line["cpu_baseline"] = None
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
