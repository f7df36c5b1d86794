"""Benchmark of photon-differential splatting forward+backward on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference|reference-gpu]
                    [--workload batch64|uniform1m|contention]

Workloads (synthetic, seeded; the reference publishes no benchmark and its photons come from
OptiX tracing, which these generators replace):
  batch64     (default) 64 independent simulations, photon counts ~ logU[2^16, 2^22]
              (45.4 M photons in all at the rank-0 seed), square images drawn from
              {256, 512, 1024}^2,
              half-uniform/half-clustered photons with differentials s ~ logU[0.5, 4] px,
              max_pixel_radius 20, fp32. One step = binning + forward + backward of every
              simulation (one Landweber iteration's splatting work) with fixed upstream
              gradients.
  uniform1m   2^20 photons on one 512^2 image (the CPU-runnable case).
  contention  2^26 photons on 2048^2, 80% on 4 sharp caustic curves, s ~ logU[0.25, 16].

Arms:
  ours           the sm_100a kernels through the C ABI; batched steps replay one CUDA graph.
  reference      the reference's splat formula on the host cores: the CPU port in
                 oracle/pds_oracle.c in the reference's float32 arithmetic (REF32 mode), all
                 host threads, on a bounded photon sample per step (the reference itself has
                 no CPU implementation of this path).
  reference-gpu  the reference's own CUDA extension (built unmodified from its sources into
                 oracle/_ref), run as the reference runs it: one pds_forward + pds_backward
                 per simulation.

Prints one JSON line (rank 0). Multi-GPU (torchrun, one process per GPU): every rank runs
its own independently seeded batch (the simulations shard with no data-path exchange), the
step time is the max over ranks, and value counts the photons of all ranks ("weak").
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from shapefromcaustics_b200 import synthetic as S  # noqa: E402

METRIC = "photon fwd+bwd splats/s"
PHASE_KERNELS = {"forward": "fwd_tiles_kernel + tail_fwd_kernel",
                 "backward": "bwd_tiles_kernel + tail_bwd_kernel + grad_scatter"}
UNIT = "photons/s"
MPR = 20
FP32_SIMT_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # 74.4, nominal (no measured figure)
# FLOPs per pixel inside the support (where the reference adds a value), counted from its formula
# (photon_differentials.cu:98-106 forward, :179-205 backward).
FLOP_FWD_PX = 22
FLOP_BWD_PX = 55


# ------------------------------------------------------------------ environment ----------

def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.isfile(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms; keeps the samples whose
    timestamps fall in the windows marked with mark_start/mark_stop."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self.windows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._reader, daemon=True)
        self.thread.start()

    def _reader(self):
        for line in self.proc.stdout:
            self.samples.append((time.time(), line.strip()))

    def mark_start(self):
        self.windows.append([time.time(), None])

    def mark_stop(self):
        self.windows[-1][1] = time.time()

    def stop(self):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        for t, line in self.samples:
            if any(a <= t <= (b or 1e300) + 0.15 for a, b in self.windows):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples in window"],
                    "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def barrier(world):
    if world > 1:
        torch.distributed.barrier()


def max_over_ranks(v, world, device):
    if world == 1:
        return v
    t = torch.tensor([v], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(v, world, device):
    if world == 1:
        return v
    t = torch.tensor([v], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.SUM)
    return float(t.item())


# ------------------------------------------------------------------ workloads ------------

def workload(name, rank, device):
    """-> (specs, concatenated photons on device, flat upstream gradient on device, desc)."""
    seed = 1000 + rank
    if name == "batch64":
        specs = S.batch_specs(64, seed=seed)
        photons = S.batch_photons(specs, seed=seed, device=device)
        desc = ("64 simulations, N_i ~ logU[2^16,2^22], images {256,512,1024}^2, "
                "uniform+cluster photons, s ~ logU[0.5,4] px, mpr 20, fp32")
    elif name == "uniform1m":
        specs = [(2 ** 20, (1, 512, 512))]
        photons = S.uniform_cluster_photons(2 ** 20, 512, 512, seed=seed, device=device)
        desc = "2^20 photons, 512^2, uniform+cluster, s ~ logU[0.5,4] px, mpr 20, fp32"
    elif name == "medium":
        specs = [(2 ** 23, (1, 1024, 1024))]
        photons = S.uniform_cluster_photons(2 ** 23, 1024, 1024, seed=seed, device=device)
        desc = "2^23 photons, 1024^2, uniform+cluster, s ~ logU[0.5,4] px, mpr 20, fp32"
    elif name in ("contention", "contention24"):
        n = 2 ** 26 if name == "contention" else 2 ** 24
        specs = [(n, (1, 2048, 2048))]
        photons = S.caustic_curve_photons(n, 2048, 2048, seed=seed, device=device)
        desc = (f"2^{n.bit_length() - 1} photons, 2048^2, 80% on 4 caustic curves (1.5 px), "
                "s ~ logU[0.25,16] px, mpr 20, fp32")
    else:
        raise SystemExit(f"unknown workload {name}")
    grads = [S.upstream_grad(shape, seed=seed * 7919 + s, device=device).reshape(-1)
             for s, (_, shape) in enumerate(specs)]
    return specs, photons, torch.cat(grads).contiguous(), desc


def split_photons(specs, photons):
    """Per-simulation contiguous copies (the plain per-simulation loop needs them)."""
    out, b = [], 0
    for n, _ in specs:
        out.append(tuple(t[..., b:b + n].contiguous() for t in photons))
        b += n
    return out


def box_pixels(specs, photons, mpr):
    """Visited box pixels per direction (the reference's loop trip count, clipped to the
    image), computed with the reference's double-precision footprint rule."""
    E, X, M, C, R = photons
    total, b = 0, 0
    for n, (_, H, W) in specs:
        x = X[0, b:b + n].double()
        y = X[1, b:b + n].double()
        r = R[b:b + n].double()
        rx = torch.clamp(torch.ceil(r * 0.5 * W), max=mpr)
        ry = torch.clamp(torch.ceil(r * 0.5 * H), max=mpr)
        pxc = torch.trunc((0.5 * x + 0.5) * W)
        pyc = torch.trunc((0.5 * y + 0.5) * H)
        w = (torch.clamp(pxc + rx, max=W - 1) - torch.clamp(pxc - rx, min=0) + 1).clamp(min=0)
        h = (torch.clamp(pyc + ry, max=H - 1) - torch.clamp(pyc - ry, min=0) + 1).clamp(min=0)
        total += float((w * h).sum().item())
        b += n
    return total


def h2d_bandwidth(device, nbytes=1 << 30, reps=3):
    """Pinned host -> device copy bandwidth (GB/s) of one large copy, best of reps."""
    host = torch.empty(nbytes // 4, dtype=torch.float32).pin_memory()
    dev = torch.empty(nbytes // 4, dtype=torch.float32, device=device)
    dev.copy_(host, non_blocking=True)
    torch.cuda.synchronize(device)
    best = None
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        dev.copy_(host, non_blocking=True)
        e1.record()
        torch.cuda.synchronize(device)
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    del host, dev
    return nbytes / (best * 1e6)


def support_pixels(specs, photons, mpr):
    """Pixels inside the kernel's support (|M d| < 1) per direction: the footprint ellipse's
    area, pi (W/2)(H/2) / |det M|, capped by its clipped box (the reference evaluates the
    whole box, but only these pixels contribute)."""
    E, X, M, C, R = photons
    total, b = 0, 0
    for n, (_, H, W) in specs:
        m = M[:, :, b:b + n].double()
        det = (m[0, 0] * m[1, 1] - m[0, 1] * m[1, 0]).abs()
        ell = math.pi * (0.5 * W) * (0.5 * H) / det.clamp(min=1e-30)
        x = X[0, b:b + n].double()
        y = X[1, b:b + n].double()
        r = R[b:b + n].double()
        rx = torch.clamp(torch.ceil(r * 0.5 * W), max=mpr)
        ry = torch.clamp(torch.ceil(r * 0.5 * H), max=mpr)
        pxc = torch.trunc((0.5 * x + 0.5) * W)
        pyc = torch.trunc((0.5 * y + 0.5) * H)
        w = (torch.clamp(pxc + rx, max=W - 1) - torch.clamp(pxc - rx, min=0) + 1).clamp(min=0)
        h = (torch.clamp(pyc + ry, max=H - 1) - torch.clamp(pyc - ry, min=0) + 1).clamp(min=0)
        total += float(torch.minimum(ell, w * h).sum().item())
        b += n
    return total


# Measured DRAM traffic per photon of each phase's kernels (ncu dram__bytes_read.sum +
# dram__bytes_write.sum on the 2^23-photon 1024^2 workload, profiles/*__medium.md), scaled to
# a workload by its photon count.
TRAFFIC_PER_PHOTON = {"plan": (309.602816e6 + 11.343360e6 + 349.815040e6 +
                               255.564032e6) / 2 ** 23,
                      "forward": (261.056000e6 + 6.905344e6) / 2 ** 23,
                      "backward": (262.672896e6 + 216.617984e6 + 327.180800e6 +
                                   263.077888e6) / 2 ** 23}


# ------------------------------------------------------------------ our arm --------------

def time_graph(graph, steps, stream):
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    with torch.cuda.stream(stream):
        ev[0].record(stream)
        for k in range(steps):
            graph.replay()
            ev[k + 1].record(stream)
    torch.cuda.synchronize()
    return [ev[k].elapsed_time(ev[k + 1]) for k in range(steps)]


def run_ours(args, rank, world, device):
    from shapefromcaustics_b200 import _lib
    from shapefromcaustics_b200.splatting import BatchedSplat, SplatPlan
    torch.cuda.set_device(device)
    specs, photons, gflat, desc = workload(args.workload, rank, device)
    n_total = sum(n for n, _ in specs)
    pixels = sum(C * H * W for _, (C, H, W) in specs)
    # the project's autotuner picks the launch configuration on this workload (untimed)
    tuned = None
    if args.config:
        tuned = json.loads(args.config)
    elif not (args.no_autotune or args.lean):
        from shapefromcaustics_b200 import autotune
        tuned, _ = autotune.tune_batch(specs, photons, gflat, MPR, device, reps=2)
    cfg = _lib.config(**tuned) if tuned else None
    batch = BatchedSplat(specs, MPR, device, config=cfg)
    out = torch.empty(batch.image_elems, device=device)
    grads = tuple(torch.empty_like(t) for t in photons[:3])
    stream = torch.cuda.Stream(device)

    def step():
        batch.plan(*photons)
        batch.forward(out)
        batch.backward(gflat, grads)

    # eager warm-up (also sets kernel attributes), then capture one graph of the whole step
    stream.wait_stream(torch.cuda.current_stream(device))
    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3)):
            step()
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        step()
    torch.cuda.synchronize()
    for _ in range(max(args.warmup, 3)):
        graph.replay()
    torch.cuda.synchronize()

    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    gpu_id = vis.split(",")[device.index].strip() if vis else str(device.index)
    clocks = ClockSampler(gpu_id)
    clocks.start()
    time.sleep(0.3)
    # ---- timed region: K graph replays ----
    barrier(world)
    torch.cuda.synchronize()
    clocks.mark_start()
    per_step = time_graph(graph, args.steps, stream)
    clocks.mark_stop()
    barrier(world)
    total_ms = max_over_ranks(sum(per_step), world, device)
    ms_per_step = total_ms / args.steps
    photons_all = sum_over_ranks(float(n_total), world, device)
    value = photons_all / (ms_per_step / 1e3)
    # error of the timed step's own outputs against the FP64 oracle (outside the timed region)
    parity = None
    if not args.lean and rank == 0:
        parity = parity_vs_oracle(specs, photons, gflat, batch, out, grads)

    # ---- roofline window: the same steps eager, CUDA events around each phase ----
    phases = {"plan": [], "forward": [], "backward": []}
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            e[0].record(stream)
            batch.plan(*photons)
            e[1].record(stream)
            batch.forward(out)
            e[2].record(stream)
            batch.backward(gflat, grads)
            e[3].record(stream)
            torch.cuda.synchronize()
            phases["plan"].append(e[0].elapsed_time(e[1]))
            phases["forward"].append(e[1].elapsed_time(e[2]))
            phases["backward"].append(e[2].elapsed_time(e[3]))
    ph_ms = {k: statistics.median(v) for k, v in phases.items()}

    if args.lean:
        clocks.stop()
        return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
                "phase_ms": ph_ms, "lean": True, "clocks": clocks.summary()}

    # ---- plain: one plan + forward + backward per simulation, like the reference's loop ----
    per_sim = split_photons(specs, photons)
    gviews = []
    b = 0
    for _, (C, H, W) in specs:
        gviews.append(gflat[b:b + C * H * W].view(C, H, W))
        b += C * H * W

    def plain_step():
        for (n, shape), ph, g in zip(specs, per_sim, gviews):
            p = SplatPlan(*ph, shape, MPR, config=cfg)
            p.forward()
            p.backward(g)

    with torch.cuda.stream(stream):
        for _ in range(2):
            plain_step()
        torch.cuda.synchronize()
        plain_steps = max(1, min(args.steps, 5))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        clocks.mark_start()
        e0.record(stream)
        for _ in range(plain_steps):
            plain_step()
        e1.record(stream)
        torch.cuda.synchronize()
        clocks.mark_stop()
    plain_ms = max_over_ranks(e0.elapsed_time(e1) / plain_steps, world, device)
    del per_sim

    # ---- parity spot check: batched vs plain forward on simulation 0 ----
    imgs = batch.images(out)
    p0 = SplatPlan(*split_photons(specs[:1], photons)[0], specs[0][1], MPR)
    ref0 = p0.forward()
    torch.cuda.synchronize()
    parity_plain = float((imgs[0] - ref0).norm() / ref0.norm())

    # ---- e2e: host (pinned) photons and gradients in, loss out, through the public API ----
    # Every step copies its photons and upstream gradient from pinned host memory and reads
    # its loss back. Two device input sets alternate, so step k+1's host->device copies (on a
    # copy stream) overlap step k's kernels; all copies lie inside the timed region.
    # Column 2 of Mp is never read by the kernels, so only Mp[:, :2] (two contiguous blocks)
    # crosses PCIe.
    host_ph = [t.cpu().pin_memory() for t in photons]
    host_g = gflat.cpu().pin_memory()
    sets = [([torch.zeros_like(t) for t in photons], torch.empty_like(gflat)) for _ in range(2)]
    loss_host = torch.empty(2, dtype=torch.float32).pin_memory()

    def copy_pairs(dev_ph):
        pairs = []
        for k, (d, h) in enumerate(zip(dev_ph, host_ph)):
            if k == 2:  # Mp [2][3][N]
                pairs += [(d[0, :2], h[0, :2]), (d[1, :2], h[1, :2])]
            else:
                pairs.append((d, h))
        return pairs

    h2d = sum(h.numel() * h.element_size() for _, h in copy_pairs(sets[0][0])) + \
        host_g.numel() * 4
    e2e_steps = max(2, min(args.steps, 6))
    copy_stream = torch.cuda.Stream(device)
    copied = [torch.cuda.Event() for _ in range(2)]
    consumed = [torch.cuda.Event() for _ in range(2)]

    def h2d_copy(k):
        dev_ph, dev_g = sets[k % 2]
        with torch.cuda.stream(copy_stream):
            copy_stream.wait_event(consumed[k % 2])
            for d, h in copy_pairs(dev_ph):
                d.copy_(h, non_blocking=True)
            dev_g.copy_(host_g, non_blocking=True)
            copied[k % 2].record(copy_stream)

    def e2e_compute(k):
        dev_ph, dev_g = sets[k % 2]
        with torch.cuda.stream(stream):
            stream.wait_event(copied[k % 2])
            batch.plan(*dev_ph)
            batch.forward(out)
            batch.backward(dev_g, grads)
            loss_host[k % 2:k % 2 + 1].copy_(torch.dot(out, dev_g).reshape(1), non_blocking=True)
            consumed[k % 2].record(stream)

    for e in consumed:
        e.record(stream)
    h2d_copy(0)
    e2e_compute(0)
    torch.cuda.synchronize()
    barrier(world)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    copy_stream.wait_stream(stream)
    h2d_copy(0)
    for k in range(e2e_steps):
        if k + 1 < e2e_steps:
            h2d_copy(k + 1)
        e2e_compute(k)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / e2e_steps, world, device)
    h2d_gbs = h2d_bandwidth(device)
    clocks.stop()

    # ---- roofline of the dominant phase ----
    peak, peak_kind = measured_peaks()
    pix_box = box_pixels(specs, photons, MPR)
    pix_sup = support_pixels(specs, photons, MPR)
    alg = {"plan": n_total * 40,
           "forward": n_total * 40 + pixels * 4,
           "backward": n_total * 76 + pixels * 4}
    flops = {"plan": 0, "forward": pix_sup * FLOP_FWD_PX, "backward": pix_sup * FLOP_BWD_PX}
    dom = max(("forward", "backward"), key=lambda k: ph_ms[k])
    # the whole step against the roofline: sum_sims [N_i 116 B + C H_i W_i 4 B 2]
    step_bytes = n_total * 116 + pixels * 8
    step_roofline = {"bound": "hbm", "kernel": "whole step (plan + forward + backward)",
                     "algorithmic_bytes": step_bytes,
                     "achieved": step_bytes / (ms_per_step / 1e3) / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": step_bytes / (ms_per_step / 1e3) / 1e9 / peak,
                     "peak_source": peak_kind,
                     # DRAM bytes the step's kernels move per photon (ncu, medium workload)
                     # against the 116 algorithmic bytes per photon
                     "traffic_per_photon": sum(TRAFFIC_PER_PHOTON.values()),
                     "traffic": sum(TRAFFIC_PER_PHOTON.values()) * n_total}
    achieved = alg[dom] / (ph_ms[dom] / 1e3) / 1e9
    simt = flops[dom] / (ph_ms[dom] / 1e3) / 1e12
    # plan: plan_pass_kernel<0> (count), bucket_reduce/top/down, plan_pass_kernel<1> (place),
    # chunk_tile_kernel; forward: fwd_tiles_kernel, tail_fwd_kernel; backward:
    # bwd_tiles_kernel, tail_bwd_kernel, grad_scatter4_kernel
    launches_per_step = 6 + 2 + 3
    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generators; photons resident in HBM)",
        "config": {"workload": f"{args.workload}: {desc}", "photons_per_gpu": n_total,
                   "simulations_per_gpu": len(specs), "image_pixels_per_gpu": pixels,
                   "max_pixel_radius": MPR, "l2": "inputs larger than L2 (no flush)",
                   "parallelism": f"simulation-sharded x{world}, no collective",
                   "mode": "batched: one CUDA graph per step (plan + fwd + bwd)",
                   "launch_config": tuned or "library default"},
        "splat_steps_per_s": {"batched": 1e3 / ms_per_step, "plain": 1e3 / plain_ms,
                              "batched_over_plain": plain_ms / ms_per_step,
                              "step": "plan + forward + backward of every simulation"},
        "phase_ms": ph_ms,
        "roofline": {"bound": "hbm", "kernel": f"{dom} phase ({PHASE_KERNELS[dom]})",
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "algorithmic_bytes": alg[dom],
                     "traffic": TRAFFIC_PER_PHOTON[dom] * n_total,
                     "traffic_source": "ncu DRAM bytes per photon on the 2^23-photon 1024^2 "
                                       "workload, scaled by photons"},
        "roofline_simt": {"kernel": dom, "achieved": simt, "peak": FP32_SIMT_NOMINAL_TFLOPS,
                          "unit": "TFLOP/s", "frac": simt / FP32_SIMT_NOMINAL_TFLOPS,
                          "peak_source": "nominal (148 SM x 128 FP32 x 2 x 1.965 GHz)",
                          "flop_count": "22 (forward) / 55 (backward) FLOP per pixel "
                                        "inside the kernel's support",
                          "support_pixels_per_step": pix_sup, "box_pixels_per_step": pix_box},
        "e2e": {"value": photons_all / (e2e_ms / 1e3), "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 4,
                "ms_per_step": e2e_ms,
                # the step's copies against this box's pinned host->device bandwidth
                "h2d_gbs": h2d / (e2e_ms * 1e6), "h2d_peak_gbs": h2d_gbs,
                "h2d_frac": (h2d / (e2e_ms * 1e6)) / h2d_gbs if h2d_gbs else None,
                "h2d_peak_source": "one 1 GiB cudaMemcpyAsync from pinned host memory, best "
                                   "of 3, measured in this run"},
        "roofline_step": step_roofline,
        "gpu_launches": launches_per_step * args.steps,
        "parity_vs_oracle": parity,
        "parity_batched_vs_plain_relL2": parity_plain,
        "clocks": clocks.summary(),
    }
    if rank == 0 and world == 1 and not args.no_plate_batch and args.workload == "batch64":
        result["landweber_plate_batch"] = run_plate_batch(args, device, args.steps, args.warmup)
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        result["reference_gpu"] = reference_gpu_subprocess(args, value)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline(specs, photons, gflat, budget_s=args.cpu_seconds)
    return result


def parity_vs_oracle(specs, photons, gflat, batch, out, grads, max_photons=2 ** 23):
    """Relative L2 error of the benchmark step's own outputs (image, grad_Ep, grad_xp,
    grad_Mp) against the FP64 oracle, over the workload's first simulations up to
    ``max_photons`` photons (errors accumulated over those simulations)."""
    import numpy as np
    from oracle import oracle as O
    torch.cuda.synchronize()
    imgs = batch.images(out)
    num = {"image": 0.0, "grad_Ep": 0.0, "grad_xp": 0.0, "grad_Mp": 0.0}
    den = dict(num)
    b = gb = 0
    sims = n_ph = 0
    t0 = time.perf_counter()
    for s, (n, shape) in enumerate(specs):
        if n_ph + n > max_photons and sims > 0:
            break
        C, H, W = shape
        sl = slice(b, b + n)
        ph = [photons[0][sl], photons[1][:, sl], photons[2][:, :, sl], photons[3][:, sl],
              photons[4][sl]]
        npy = [t.cpu().numpy() for t in ph]
        G = gflat[gb:gb + C * H * W].view(C, H, W).cpu().double().numpy()
        rimg = O.forward(*npy, shape, MPR)
        rg = O.backward(G, *npy, MPR)
        got = [imgs[s].cpu().double().numpy(), grads[0][sl].cpu().double().numpy(),
               grads[1][:, sl].cpu().double().numpy(), grads[2][:, :, sl].cpu().double().numpy()]
        for k, a, r in zip(num, got, [rimg, *rg]):
            num[k] += float(np.sum((a - r) ** 2))
            den[k] += float(np.sum(r ** 2))
        b += n
        gb += C * H * W
        sims += 1
        n_ph += n
    res = {k: (num[k] / den[k]) ** 0.5 if den[k] > 0 else 0.0 for k in num}
    res.update({"metric": "relative L2 vs FP64 oracle", "simulations": sims, "photons": n_ph,
                "tolerance": {"image": 1e-5, "gradients": 1e-4},
                "oracle_seconds": round(time.perf_counter() - t0, 2)})
    return res


def reference_gpu_subprocess(args, our_value):
    """The reference's own CUDA extension on the same workload (``--impl reference-gpu`` in a
    child process, after this arm's timing); -> its value, step time and clocks."""
    cmd = [sys.executable, os.path.abspath(__file__), "--impl", "reference-gpu", "--workload",
           args.workload, "--steps", str(max(3, min(args.steps, 10))), "--warmup", "2"]
    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "LOCAL_WORLD_SIZE"):
        env.pop(k, None)
    try:
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env)
        line = [l for l in p.stdout.splitlines() if l.startswith("{")][-1]
        r = json.loads(line)
    except Exception as e:  # the reference extension may be absent (not built here)
        return {"unavailable": f"reference-gpu arm failed: {type(e).__name__}: {e}"}
    if "unavailable" in r:
        return r
    return {"value": r["value"], "unit": r["unit"], "ms_per_step": r["ms_per_step"],
            "steps": r["steps"], "clocks": r.get("clocks"), "mode": r["config"]["mode"],
            "ours_over_reference_gpu": our_value / r["value"]}


# ------------------------------------------------------------------ CPU (reference) ------

def cpu_sample(specs, photons, gflat, target):
    """A bounded sample of the workload: the first simulations' photons up to `target`."""
    take, b, gb = [], 0, 0
    got = 0
    for n, shape in specs:
        C, H, W = shape
        k = min(n, target - got)
        if k <= 0:
            break
        take.append((k, shape, b, gb))
        got += k
        b += n
        gb += C * H * W
    return take


def cpu_run(take, photons_cpu, g_cpu, threads, mode="ref32"):
    from oracle import oracle as O
    E, X, M, C, R = photons_cpu
    t0 = time.perf_counter()
    n = 0
    for k, shape, b, gb in take:
        sl = slice(b, b + k)
        Cc, H, W = shape
        G = g_cpu[gb:gb + Cc * H * W].reshape(Cc, H, W).double().numpy()
        args = (E[sl].numpy(), X[:, sl].numpy(), M[:, :, sl].numpy(), C[:, sl].numpy(), R[sl].numpy())
        O.forward(*args, shape, MPR, mode=mode, threads=threads)
        O.backward(G, *args, MPR, mode=mode, threads=threads)
        n += k
    return n, time.perf_counter() - t0


def cpu_baseline(specs, photons, gflat, budget_s=15.0):
    threads = os.cpu_count() or 1
    photons_cpu = [t.cpu() for t in photons]
    g_cpu = gflat.cpu()
    # size the sample from a short probe so the timed CPU run takes about budget_s
    probe = cpu_sample(specs, photons_cpu, g_cpu, 2 ** 17)
    n, dt = cpu_run(probe, photons_cpu, g_cpu, threads)
    target = int(max(2 ** 17, min(sum(n for n, _ in specs), n / max(dt, 1e-3) * budget_s)))
    take = cpu_sample(specs, photons_cpu, g_cpu, target)
    # the whole workload may take less than the budget: repeat it (at least 10 s of work)
    n, dt, passes = 0, 0.0, 0
    while passes < 8 and (passes == 0 or dt < min(10.0, budget_s)):
        ni, di = cpu_run(take, photons_cpu, g_cpu, threads)
        n, dt, passes = n + ni, dt + di, passes + 1
    return {"value": n / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"first {n // passes} photons of the workload ({len(take)} simulations) "
                      f"x {passes} passes, fwd+bwd, reference float32 arithmetic, {dt:.1f} s"}


def run_reference_cpu(args, rank, world):
    if rank != 0:
        return None
    sample = int(args.ref_sample)
    specs, photons, gflat, desc = workload_cpu(args.workload, sample)
    threads = os.cpu_count() or 1
    take = cpu_sample(specs, photons, gflat, sample)
    for _ in range(args.warmup):
        cpu_run(take[:1], photons, gflat, threads)
    times, n = [], 0
    for _ in range(args.steps):
        n, dt = cpu_run(take, photons, gflat, threads)
        times.append(dt)
    ms = 1e3 * sum(times) / len(times)
    value = n / (ms / 1e3)
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": f"{args.workload}: {desc}", "max_pixel_radius": MPR,
                       "sample_photons_per_step": n},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{n} photons per step (first simulations of the "
                                       f"workload), fwd+bwd, reference float32 arithmetic"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def workload_cpu(name, target):
    """The workload's leading simulations (enough for `target` photons), drawn on the CPU."""
    if name != "batch64":
        specs, photons, gflat, desc = workload(name, 0, "cpu")
        return specs, photons, gflat, desc
    seed = 1000
    specs_all = S.batch_specs(64, seed=seed)
    specs, got = [], 0
    for sp in specs_all:
        if got >= target:
            break
        specs.append(sp)
        got += sp[0]
    parts = [S.uniform_cluster_photons(n, H, W, seed=seed * 1000003 + s, device="cpu")
             for s, (n, (C, H, W)) in enumerate(specs)]
    photons = tuple(torch.cat([p[k] for p in parts], dim=-1).contiguous() for k in range(5))
    grads = [S.upstream_grad(shape, seed=seed * 7919 + s).reshape(-1)
             for s, (_, shape) in enumerate(specs)]
    desc = ("64 simulations, N_i ~ logU[2^16,2^22], images {256,512,1024}^2, "
            "uniform+cluster photons, s ~ logU[0.5,4] px, mpr 20, fp32")
    return specs, photons, torch.cat(grads), desc


def run_reference_gpu(args, rank, world, device):
    try:
        from oracle import build_ref
        ref = build_ref.load_module()
    except Exception as e:
        return {"impl": "reference-gpu", "unavailable": f"reference extension not built: {e}"}
    torch.cuda.set_device(device)
    specs, photons, gflat, desc = workload(args.workload, rank, device)
    n_total = sum(n for n, _ in specs)
    per_sim = split_photons(specs, photons)
    gviews, b = [], 0
    for _, (C, H, W) in specs:
        gviews.append(gflat[b:b + C * H * W].view(C, H, W))
        b += C * H * W

    def step():
        for (n, shape), ph, g in zip(specs, per_sim, gviews):
            ref.pds_forward(*ph, list(shape), MPR)
            ref.pds_backward(g, *ph, MPR)

    for _ in range(max(args.warmup, 1)):
        step()
    torch.cuda.synchronize()
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    clocks = ClockSampler(vis.split(",")[device.index].strip() if vis else str(device.index))
    clocks.start()
    time.sleep(0.3)
    barrier(world)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    clocks.mark_start()
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    clocks.mark_stop()
    clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world, device)
    photons_all = sum_over_ranks(float(n_total), world, device)
    return {"metric": METRIC, "value": photons_all / (ms / 1e3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference-gpu", "clocks": clocks.summary(),
            "config": {"workload": f"{args.workload}: {desc}", "max_pixel_radius": MPR,
                       "mode": "plain: pds_forward + pds_backward per simulation"}}


# ------------------------------------------------------------------ Landweber workloads --

def plate_setup(n_field, image, per_texel, device, seed=0, texel=0.1, dist=50.0, amp=0.05):
    """Height-field plate of the Landweber workloads: a 1 mm base plus 32 Gaussian bumps
    (amplitude U[0, amp] mm, 50 um by default, width U[4, 24] texels), collimated light at
    normal incidence, n = 1.5, receiver 50 mm below; photons jittered per texel."""
    from shapefromcaustics_b200 import scene as SC
    half = 0.5 * n_field * texel * 1.1
    scene = SC.PlateScene(texel=texel, ior=1.5, receiver_distance=dist, receiver_half=half)
    h = SC.height_field_bumps(n_field, n_field, seed=seed, bumps=32, base=1.0,
                              amp=(0.0, amp), width=(4.0, 24.0)).float().to(device)
    t = SC.height_field_bumps(n_field, n_field, seed=seed + 1, bumps=32, base=1.0,
                              amp=(0.0, amp), width=(4.0, 24.0)).float().to(device)
    return scene, h, t


def plate_batch_setup(device, seed=1000, n_sims=64, n_field=256, footprint_px=3.0):
    """The uneven batch of Landweber simulations: one 256^2 height field (the 256^2 Landweber
    workload's generator), 64 simulations with the batch's photon counts ~ logU[2^16, 2^22]
    (rounded to whole photons per texel) and image sizes {256, 512, 1024}^2, each with its own
    light tilt (up to 5 degrees, uniform azimuth) and wavelength (U[450, 650] nm, the fused
    silica index at it); initial footprints of footprint_px receiver pixels."""
    import numpy as np
    from shapefromcaustics_b200 import plate as PL
    from shapefromcaustics_b200 import scene as SC
    scene, h_true, h_tgt = plate_setup(n_field, 512, 4, device, seed=0)
    rng = np.random.default_rng(seed)
    specs = S.batch_specs(n_sims, seed=seed)
    sims, per_texel = [], []
    for n, shape in specs:
        per = max(1, int(round(n / float(n_field * n_field))))
        th, ph = np.radians(5.0) * rng.random(), 2 * np.pi * rng.random()
        light = (np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), -np.cos(th))
        lam = 0.45 + 0.2 * rng.random()
        s = SC.PlateScene(texel=scene.texel, ior=float(SC.fused_silica(lam)),
                          receiver_distance=scene.receiver_distance,
                          receiver_half=scene.receiver_half, light_dir=light)
        p = PL.plate_params(s, footprint_px * 2.0 * s.receiver_half / shape[1])
        sims.append((per * n_field * n_field, shape, p))
        per_texel.append(per)
    return scene, h_true, h_tgt, sims, per_texel


def check_refract_backward(batch, h, px, py, flux, gh):
    """The batched refraction backward alone (the last step of BatchedPlate.backward), from
    the gradient records the splat backward left in the plan's workspace."""
    import ctypes
    from shapefromcaustics_b200._lib import check, lib
    from shapefromcaustics_b200.splatting import _ptr, _stream
    sp = batch.splat
    with torch.cuda.device(batch.device):
        check(lib().pds_batch_refract_backward_planned_f32(
            _ptr(h), h.shape[0], h.shape[1], _ptr(batch.plates_dev), _ptr(batch.begins_dev),
            batch.n_sims, _ptr(px), _ptr(py), _ptr(flux), batch.n_total, sp.n_tiles,
            _ptr(sp.ws), sp.ws.numel(), ctypes.byref(sp.cfg), _ptr(gh), _stream(batch.device)))


def run_plate_batch(args, device, steps, warmup, config=None):
    """One Landweber iteration over the uneven batch of simulations with refraction
    (plate_batch_setup), batched (one CUDA graph: photon sources, one batched refraction, one
    splat plan / forward / backward, one batched refraction backward, the fused update) against
    plain (the reference's per-simulation loop, shape_from_caustics.py:351-353: each
    simulation's source, refraction, plan, forward, backward and refraction backward launched
    in turn from Python). -> dict of iterations per second and the batch's size."""
    from shapefromcaustics_b200 import plate as PL
    from shapefromcaustics_b200.landweber import LandweberParams, landweber_update, photon_source
    from shapefromcaustics_b200.splatting import SplatPlan
    scene, h_true, h_tgt, sims, per_texel = plate_batch_setup(device)
    nf = h_true.shape[0]
    from shapefromcaustics_b200 import _lib
    batch = PL.BatchedPlate(sims, MPR, device,
                            config=_lib.config(**config) if config else None)
    n_total = batch.n_total
    px = torch.empty(n_total, device=device)
    py = torch.empty(n_total, device=device)
    flux = torch.cat([torch.full((n,), 1.0 / n, device=device) for n, _, _ in sims])
    views, b = [], 0
    for n, _, _ in sims:
        views.append((px[b:b + n], py[b:b + n], flux[b:b + n]))
        b += n

    def sources(offset0):
        off = offset0
        for per, (vx, vy, _) in zip(per_texel, views):
            _, _, off = photon_source(nf, nf, per, scene.texel, 7, off, device, out=(vx, vy))
        return off

    sources(0)
    target = batch.forward(h_tgt.contiguous(), px, py, flux).clone()
    base = 1.0
    d0 = (h_true - base).clone()
    d = d0.clone()
    h = (base + d).contiguous()
    mask = torch.ones_like(d)
    vol = float(d.sum())
    params = LandweberParams(tau=1e-4, d1=0.75 * vol, d2=1.25 * vol)
    ws = torch.empty(1 << 22, dtype=torch.uint8, device=device)
    img = torch.empty(batch.image_elems, device=device)
    gimg = torch.empty_like(img)
    gh = torch.zeros_like(d)

    # Every timed iteration starts from the same field (the true one): the iterations are
    # timed, not the trajectory, and a step size that carried the field away (to the update's
    # clamp bounds, with folded caustics and footprints at the radius cap) would time a
    # different workload at every step.
    def batched_step():
        d.copy_(d0)
        torch.add(d, base, out=h)
        sources(0)
        batch.forward(h, px, py, flux, out=img)
        torch.sub(img, target, out=gimg)
        gh.zero_()
        batch.backward(h, px, py, flux, gimg, grad_height=gh)
        landweber_update(d, gh, mask, params, ws)
        torch.add(d, base, out=h)

    t_views = batch.images(target)

    def plain_step():
        d.copy_(d0)
        torch.add(d, base, out=h)
        gh.zero_()
        off = 0
        for k, ((n, shape, p), per, (vx, vy, vf)) in enumerate(zip(sims, per_texel, views)):
            _, _, off = photon_source(nf, nf, per, scene.texel, 7, off, device, out=(vx, vy))
            inputs = PL.refract_forward(h, vx, vy, vf, p)
            plan = SplatPlan(*inputs, shape, MPR)
            g = plan.forward() - t_views[k]
            plan.backward(g, records=True)
            PL.refract_backward_planned(h, vx, vy, vf, p, plan, grad_height=gh)
        landweber_update(d, gh, mask, params, ws)
        torch.add(d, base, out=h)

    stream = torch.cuda.Stream(device)
    stream.wait_stream(torch.cuda.current_stream(device))
    with torch.cuda.stream(stream):
        for _ in range(max(warmup, 3)):
            batched_step()
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        batched_step()
    torch.cuda.synchronize()
    for _ in range(max(warmup, 3)):
        graph.replay()
    torch.cuda.synchronize()
    per = time_graph(graph, steps, stream)
    ms_b = sum(per) / steps
    with torch.cuda.stream(stream):
        for _ in range(2):
            plain_step()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        k = max(2, min(steps, 5))
        e0.record(stream)
        for _ in range(k):
            plain_step()
        e1.record(stream)
        torch.cuda.synchronize()
    ms_p = e0.elapsed_time(e1) / k
    del graph
    # phases of the batched step (eager, CUDA events on the stream)
    names = ["sources", "refract_fwd", "plan", "splat_fwd", "data_grad", "splat_bwd",
             "refract_bwd", "update"]
    acc = {k: [] for k in names}
    splat = batch.splat
    with torch.cuda.stream(stream):
        for rep in range(3):
            d.copy_(d0)
            torch.add(d, base, out=h)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(len(names) + 1)]
            ev[0].record(stream)
            sources(0)
            ev[1].record(stream)
            inputs = batch._inputs(h, px, py, flux)
            ev[2].record(stream)
            splat.plan(*inputs)
            ev[3].record(stream)
            splat.forward(img)
            ev[4].record(stream)
            torch.sub(img, target, out=gimg)
            ev[5].record(stream)
            splat.backward(gimg, records=True)  # the forward's splat inputs, kept
            ev[6].record(stream)
            gh.zero_()
            check_refract_backward(batch, h, px, py, flux, gh)
            ev[7].record(stream)
            landweber_update(d, gh, mask, params, ws)
            ev[8].record(stream)
            torch.cuda.synchronize()
            for k, nm in enumerate(names):
                acc[nm].append(ev[k].elapsed_time(ev[k + 1]))
    phases = {k: statistics.median(v) for k, v in acc.items()}
    return {"batched_it_per_s": 1e3 / ms_b, "plain_it_per_s": 1e3 / ms_p,
            "batched_over_plain": ms_p / ms_b, "batched_ms": ms_b, "plain_ms": ms_p,
            "batched_phase_ms": phases,
            "photons_per_iteration": n_total, "simulations": len(sims),
            "workload": "uneven batch with refraction: 256^2 height field, 64 simulations, "
                        "N_i ~ logU[2^16, 2^22] (whole photons per texel), images "
                        "{256,512,1024}^2, light tilt <= 5 deg, wavelength U[450,650] nm "
                        "(fused silica), 3-pixel footprints; one Landweber iteration "
                        "(sources, refraction, splat, backward, update), each from the true "
                        "field",
            "batched": "one CUDA graph: 64 source launches, one batched refraction, one plan / "
                       "forward / backward, one batched refraction backward, the update; the "
                       "refracted splat inputs kept from forward to backward",
            "plain": "per simulation from Python: source, refraction, plan, forward, "
                     "backward, refraction backward; then the update"}


def run_landweber_step(args, rank, world, device):
    """One Landweber iteration on a 256^2 field, 4 photons per texel (262,144), 512^2
    image: refraction + splat forward, L2 discrepancy against a target rendered from a second
    field, backward through splat and refraction, fused projected update."""
    from shapefromcaustics_b200.landweber import LandweberParams, jitter, landweber_update
    from shapefromcaustics_b200.plate import PlateSplat, plate_params
    torch.cuda.set_device(device)
    nf, img, pt = 256, 512, 4
    scene, h_true, h_tgt = plate_setup(nf, img, pt, device)
    n = nf * nf * pt
    du0 = 3.0 * 2.0 * scene.receiver_half / img  # 3-pixel initial footprint
    pp = plate_params(scene, du0)
    g = torch.Generator(device=device)
    g.manual_seed(rank)
    px, py = jitter(nf, nf, scene, pt, g, device)
    flux = torch.full((n,), 1.0 / n, device=device)
    shape = (1, img, img)
    with torch.no_grad():
        target = PlateSplat.apply(h_tgt, px, py, flux, pp, shape, MPR, False)
    base = 1.0
    d0 = (h_true - base).clone()
    d = d0.clone()
    mask = torch.ones_like(d)
    vol = float(d.sum())
    params = LandweberParams(d1=0.75 * vol, d2=1.25 * vol)
    tn = float((target * target).sum())
    ws = torch.empty(1 << 22, dtype=torch.uint8, device=device)
    def step():
        # every iteration from the same field (see run_plate_batch)
        d.copy_(d0)
        hv = (base + d).requires_grad_(True)
        im = PlateSplat.apply(hv, px, py, flux, pp, shape, MPR, True)
        loss = 0.5 * ((im - target) ** 2).sum() / tn
        loss.backward()
        landweber_update(d, hv.grad, mask, params, ws)

    stream = torch.cuda.Stream(device)
    stream.wait_stream(torch.cuda.current_stream(device))
    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3)):
            step()
    torch.cuda.synchronize()
    # eager iterations (each op launched from Python through autograd), then the same
    # iteration captured once in a CUDA graph and replayed
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier(world)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
    torch.cuda.synchronize()
    ms_eager = max_over_ranks(e0.elapsed_time(e1) / args.steps, world, device)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        step()
    torch.cuda.synchronize()
    for _ in range(max(args.warmup, 3)):
        graph.replay()
    torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(sum(time_graph(graph, args.steps, stream)) / args.steps, world, device)
    # the replayed iteration's update against an eager one from the same field
    with torch.cuda.stream(stream):
        graph.replay()
        d_graph = d.clone()
        step()
    torch.cuda.synchronize()
    graph_vs_eager = float((d_graph - d).norm() / max(float((d - d0).norm()), 1e-30))
    del graph
    its = sum_over_ranks(1.0, world, device) / (ms / 1e3)
    return {"metric": "Landweber it/s", "value": its, "unit": "it/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "landweber256: 256^2 height field (1 mm + 32 bumps), 4 "
                                   "jittered photons/texel (262144), n=1.5, receiver 50 mm, "
                                   "512^2 image, L2 vs second field; refraction + splat "
                                   "fwd/bwd + fused update; each iteration from the true "
                                   "field", "photons": n,
                       "launch_config": "library default",
                       "mode": "one CUDA graph per iteration (autograd forward, backward and "
                               "update captured once)"},
            "eager_it_per_s": 1e3 / ms_eager, "eager_ms_per_step": ms_eager,
            "graph_vs_eager_update_relL2": graph_vs_eager}


def run_reconstruction(args, rank, world, device):
    """Full reconstruction: 1024^2 field, 16 simulations x 4 photons per texel (2^22 each,
    67M per iteration) into a 1024^2 image, Landweber iterations (the plan and the refracted
    splat inputs kept from forward to backward unless --recon-lean); final height RMSE, peak
    HBM and the CUDA-event time of each phase of one iteration."""
    from shapefromcaustics_b200.landweber import LandweberParams, iteration_phases, reconstruct
    torch.cuda.set_device(device)
    nf = 1024
    scene, h_true, _ = plate_setup(nf, nf, 4, device, seed=7, amp=args.recon_amplitude)
    d_true = h_true - 1.0
    vol = float(d_true.sum())
    params = LandweberParams(tau=args.recon_tau, d1=0.75 * vol, d2=1.25 * vol)
    iters = args.steps
    sims = args.recon_sims
    # warm-up: a short reconstruction of its own (the allocator's first device allocations
    # and the kernels' first launches stay out of the timed run)
    warm = max(args.warmup, 3)
    res_w = reconstruct(h_true, 1.0, scene, iterations=warm, sims=sims, per_texel=4, image=nf,
                        footprint_px=args.recon_footprint, params=params, seed=rank + 1000,
                        keep_plan=not args.recon_lean, objective=args.recon_objective)
    # the target image (the reference loads it; here it is rendered from the true field) is
    # made once, outside the timed iterations
    target = res_w["target"]
    torch.cuda.synchronize()
    torch.cuda.reset_peak_memory_stats(device)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    res = reconstruct(h_true, 1.0, scene, iterations=iters, sims=sims, per_texel=4, image=nf,
                      footprint_px=args.recon_footprint, params=params, seed=rank,
                      keep_plan=not args.recon_lean, log_every=max(iters // 10, 1),
                      objective=args.recon_objective, target=target)
    t1.record()
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    peak = torch.cuda.max_memory_allocated(device)
    # the phases of an iteration at the start (flat field), whatever the step size did later
    phases = iteration_phases(1.0, res["target"], scene, torch.zeros_like(h_true),
                              torch.ones_like(h_true), params, sims=sims, per_texel=4, image=nf,
                              footprint_px=args.recon_footprint, seed=rank + 99,
                              objective=args.recon_objective, keep_plan=not args.recon_lean)
    return {"metric": "Landweber it/s", "value": iters / (ms / 1e3), "unit": "it/s",
            "n_gpus": world, "steps": iters, "warmup": warm, "ms_per_step": ms / iters,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": f"recon1024: 1024^2 field, {sims} sims x 2^22 photons per "
                                   "iteration into 1024^2",
                       "photons_per_iteration": res["photons_per_iteration"],
                       "objective": args.recon_objective, "tau": args.recon_tau,
                       "bump_amplitude_mm": args.recon_amplitude,
                       "kept_for_backward": "recomputed" if args.recon_lean else
                       "plan and refracted splat inputs",
                       "footprint_px": args.recon_footprint},
            "final_height_rmse_mm": res["rmse"],
            "initial_height_rmse_mm": float((d_true ** 2).mean().sqrt()),
            "rmse_history": res["history"]["rmse"],
            "discrepancy_history": res["history"]["discrepancy"],
            "phase_ms": phases,
            "peak_hbm_bytes": peak}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference-gpu"])
    ap.add_argument("--workload", default="batch64",
                    choices=["batch64", "uniform1m", "medium", "contention", "contention24",
                             "landweber256", "recon1024"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plate-batch", action="store_true",
                    help="skip the batched-vs-plain Landweber iteration with refraction")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip the reference CUDA extension's run on the same workload")
    ap.add_argument("--no-autotune", action="store_true",
                    help="time the library's default configuration instead of the tuned one")
    ap.add_argument("--lean", action="store_true",
                    help="timed steps and phase timings only, default configuration "
                         "(for profiler runs)")
    ap.add_argument("--config", default=None,
                    help="launch configuration as JSON pds_config fields (skips the autotuner)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-sample", type=float, default=2 ** 21)
    ap.add_argument("--recon-objective", default="l2_sq", choices=["l2_sq", "normalized"],
                    help="recon1024: the reference's 0.5 |I - T|^2 or it divided by |T|^2")
    ap.add_argument("--recon-tau", type=float, default=1e-7,
                    help="recon1024: gradient step (the reference's tau_pixel; its default "
                         "0.1 diverges on this scene with the l2_sq data term)")
    ap.add_argument("--recon-sims", type=int, default=16,
                    help="recon1024: simulations per iteration (2^22 photons each)")
    ap.add_argument("--recon-amplitude", type=float, default=0.05,
                    help="recon1024: largest bump amplitude of the true field (mm)")
    ap.add_argument("--recon-lean", action="store_true",
                    help="recon1024: recompute the refraction and the plan in the backward "
                         "instead of keeping them (less memory)")
    ap.add_argument("--recon-footprint", type=float, default=3.0,
                    help="recon1024: initial photon footprint in receiver pixels")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    rank, world, local = dist_env()
    if args.impl == "reference":
        if world > 1:
            import datetime
            torch.distributed.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
        res = run_reference_cpu(args, rank, world)
        if world > 1:
            torch.distributed.destroy_process_group()
        if rank == 0:
            print(json.dumps(res))
        return
    device = torch.device("cuda", local)
    if world > 1:
        import datetime
        torch.cuda.set_device(device)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=device)
    if args.impl == "reference-gpu":
        res = run_reference_gpu(args, rank, world, device)
    elif args.workload == "landweber256":
        res = run_landweber_step(args, rank, world, device)
    elif args.workload == "recon1024":
        res = run_reconstruction(args, rank, world, device)
    else:
        res = run_ours(args, rank, world, device)
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(res))


if __name__ == "__main__":
    main()
