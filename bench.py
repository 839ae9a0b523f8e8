"""Benchmark of the stereo-depth hot path on the raw 1280x1024, D=128 workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--frames B]

Workload (one "step" = B frames): raw (unrectified) 1280x1024 u8 IR pairs of seeded synthetic scenes
(20 random boxes and cylinders at 200-600 mm before a back wall, speckle projector, sigma 2 DN) from one
synthetic calibration (f 1100 px, k1 -0.08, k2 0.02, right camera yawed 1.5 deg, baseline 60 mm):
GPU remap with float32 tables -> census 5x5 -> 4-path SGM (P1 8, adaptive P2 96, slant steps) with
D=128 -> WTA + subpixel -> L-R check 1 px -> 3x3 median -> depth. Metric: Gpix*disp/s = sum(W*H*D)/time.

Printed as one JSON line by rank 0:
  value          whole-job throughput, inputs resident in HBM, device-timed (CUDA events), max over ranks
  e2e            the same through the public host API (OfflineRedepth over StereoBatch): host->device copy of
                 every step's raw pairs and device->host copy of their u16 disparity + f32 depth inside the
                 timed region (double-buffered across steps), device-timed
  e2e_plugin     the drop-in call (ds_compute_raw), one frame per synchronous call from pinned host memory to
                 pinned host memory, host-clock latency p50 / p99
  frame_ms       per-frame device time percentiles (stage events)
  roofline       the dominant kernel (SGM paths) against the measured HBM copy bandwidth
  cpu_baseline   the reference CPU path (oracle/_ref: the reference's stereo.cpp) on this host's cores
  serving, batch64, offline
                 on one GPU (unless --no-extras): configuration 4 (request server, Poisson arrivals, latency
                 percentiles), configuration 3 (64 uneven pairs, batched against per-frame launches) and
                 configuration 5 (offline 8-path D=256 re-depth of a 64-frame synthetic recording)
With --impl reference, the reference CPU implementation alone is timed (rank 0 only).
Multi-GPU: independent replicas (frames shard across ranks, no collective on the data path).
"""
from __future__ import annotations

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

W, H, D, P = 1280, 1024, 128, 4
METRIC = "SGM Gpix*disp/s at 1280x1024 D=128 (batched vs per-frame; p50/p99 frame ms)"
UNIT = "Gpix*disp/s"
WORKLOAD = ("raw 1280x1024 u8 stereo pair: GPU remap (f32 tables, bilinear) + census 5x5 + 4-path SGM "
            "(P1 8, adaptive P2 96, slant) D=128 + WTA/subpixel + L-R 1 px + 3x3 median + depth")
PX_D = W * H * D


def algorithmic_bytes(w, h, d, p, c_b=1, raw=True):
    """Bytes per pair of the materialised-volume dataflow: W*H*(D*(c_b(1+P)+4P) + 66 [+20 raw])."""
    return w * h * (d * (c_b * (1 + p) + 4 * p) + 66 + (20 if raw else 0))


def path_stage_bytes(w, h, d, p, c_b=1):
    """The SGM-path share of that formula: cost reads P*c_b, first-path sum write 2 B, (P-1) RMW of 4 B."""
    return w * h * d * (p * c_b + 2 + 4 * (p - 1))


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 100 ms from warm-up to the end of the e2e run."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
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


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def replica_seed0(rank: int) -> int:
    """First scene seed of rank `rank`'s frames: replicas render disjoint scenes (no data-path collective)."""
    return 100 * rank


def max_over_ranks(v: float, world: int, device) -> float:
    """The slowest rank's time (or any per-rank value): one all-reduce MAX in float64 over the job."""
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def make_frames(n, seed0, device):
    from open_source_einstar_b200 import synth
    pairs = [synth.raw_objects_pair(seed=seed0 + i, device=device) for i in range(n)]
    return pairs


def reference_frame(ref, pair, threads_note=None):
    """The reference CPU path on one raw pair: restated calib::remap x2, the reference's sgm_disparity and
    median3 (oracle/_ref), restated depth."""
    from oracle.oracle import OracleSgm
    (lx, ly), (rx, ry) = pair.maps
    p = OracleSgm(min_disparity=pair.min_disparity, num_disparities=D)
    t0 = time.perf_counter()
    rl, rr = ref.remap(pair.left, lx, ly), ref.remap(pair.right, rx, ry)
    d = ref.median3(ref.sgm_disparity(rl, rr, p))
    ref.encode_u16(d, p.min_disparity)
    ref.depth(d, pair.f, pair.baseline, 0.0, 150.0, 700.0)
    return time.perf_counter() - t0


def cpu_reference_sample(pairs, budget_s=20.0, max_frames=8):
    from oracle.oracle import Ref
    ref = Ref()
    reference_frame(ref, pairs[0])  # warm-up (thread pool, page faults)
    times = []
    t_start = time.perf_counter()
    i = 0
    while i < max_frames and (time.perf_counter() - t_start) < budget_s:
        times.append(reference_frame(ref, pairs[i % len(pairs)]))
        i += 1
    med = statistics.median(times)
    return {"value": PX_D / med / 1e9, "unit": UNIT, "cores": ref.threads(), "kind": "reference",
            "sample": f"{len(times)} full raw 1280x1024 D=128 frames (median {med * 1e3:.0f} ms/frame): reference "
                      "libs/depth/src/stereo.cpp sgm_disparity + median3 (oracle/_ref, std::thread TBB stand-in over "
                      f"{ref.threads()} threads) + restated remap x2 and depth",
            "ms_per_frame": med * 1e3}


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    pairs = make_frames(2, replica_seed0(rank), "cpu")  # the scenes the GPU arm's first frames render
    from oracle.oracle import Ref
    ref = Ref()
    for i in range(args.warmup):
        reference_frame(ref, pairs[i % 2])
    times = []
    deadline = time.perf_counter() + args.reference_budget
    for i in range(args.steps):
        times.append(reference_frame(ref, pairs[i % 2]))
        if time.perf_counter() > deadline:
            break
    total = sum(times)
    v = len(times) * PX_D / total / 1e9
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": len(times),
            "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "frames_per_step": 1, "path": "reference CPU (one frame per step)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": ref.threads(), "kind": "reference",
                             "sample": "one full raw frame per step: reference stereo.cpp sgm_disparity + median3 "
                                       "(oracle/_ref) + restated remap and depth, all host threads"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---- serving workload: Poisson arrivals of mixed frames through the request server ---------------------------
SERVE_SIZES = (((1280, 1024), 0.7), ((960, 768), 0.2), ((640, 512), 0.1))
SERVE_RIGS = ({"f": 1100.0, "baseline": 60.0, "k1": -0.08, "k2": 0.02, "yaw_deg": 1.5},
              {"f": 1000.0, "baseline": 55.0, "k1": -0.06, "k2": 0.015, "yaw_deg": 1.2},
              {"f": 1200.0, "baseline": 65.0, "k1": -0.10, "k2": 0.03, "yaw_deg": 1.8},
              {"f": 1050.0, "baseline": 50.0, "k1": -0.07, "k2": 0.02, "yaw_deg": 1.0})
SERVE_D = (96, 128)


def serving_calibrations(dev):
    """4 synthetic rigs x 3 sizes: raw speckle pairs of boxes/cylinders at 200-600 mm with their remap tables."""
    from open_source_einstar_b200 import synth
    cal = []
    for r, rig in enumerate(SERVE_RIGS):
        for s, ((w, h), _) in enumerate(SERVE_SIZES):
            sc = w / 1280.0
            pr = synth.raw_objects_pair(seed=500 + 3 * r + s, width=w, height=h, f=rig["f"] * sc, baseline=rig["baseline"],
                                        k1=rig["k1"], k2=rig["k2"], yaw_deg=rig["yaw_deg"], num_disparities=128,
                                        device=dev)
            cal.append((r, s, w, h, pr))
    return cal


def serving_requests(cal, n, seed):
    """n request descriptors: rig uniform, size 70/20/10 %, D in {96, 128}; pinned inputs and outputs."""
    from open_source_einstar_b200 import SgmParams, StereoParams
    from open_source_einstar_b200.serving import pinned_copy, pinned_empty
    rng = np.random.default_rng(seed)
    pinned = {}
    reqs = []
    for i in range(n):
        r = int(rng.integers(len(SERVE_RIGS)))
        s = int(rng.choice(len(SERVE_SIZES), p=[p for _, p in SERVE_SIZES]))
        d = int(rng.choice(SERVE_D))
        ci = 3 * r + s
        _, _, w, h, pr = cal[ci]
        if ci not in pinned:
            pinned[ci] = (pinned_copy(pr.left), pinned_copy(pr.right))
        sp = StereoParams(sgm=SgmParams(min_disparity=pr.min_disparity, num_disparities=d))
        reqs.append({"left": pinned[ci][0], "right": pinned[ci][1], "width": w, "height": h, "params": sp, "calib": ci,
                     "outputs": {"disparity_u16": pinned_empty((h, w), np.uint16), "depth": pinned_empty((h, w), np.float32)},
                     "px_d": w * h * d})
    return reqs


def run_serving(args, world, rank, local):
    """Poisson arrivals at each rate for --duration seconds through StereoServer (ds_server_*): latency
    p50/p99/p99.9 from submit to results in host memory, beside frames/s. One GPU; replicas beyond."""
    import torch
    torch.cuda.set_device(local)
    line = serving_line(torch.device("cuda", local), args.rates, args.duration, args.slots, world, rank)
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def serving_line(dev, rates, duration, slots, world=1, rank=0):
    """The serving workload's JSON line (configuration 4) on device `dev`."""
    import torch
    from open_source_einstar_b200 import RectifiedGeometry, RemapTable
    from open_source_einstar_b200.serving import StereoServer, latency_summary, poisson_arrivals, replay
    cal = serving_calibrations(dev)
    reqs = serving_requests(cal, 512, seed=11 + rank)
    srv = StereoServer(volume_budget_bytes=40 << 30, max_slots=slots)
    for ci, (r, s, w, h, pr) in enumerate(cal):
        (lx, ly), (rx, ry) = pr.maps
        srv.add_calibration(ci, RemapTable(lx, ly), RemapTable(rx, ry), w, h,
                            RectifiedGeometry(pr.f, 0, 0, pr.baseline, pr.cx_offset), 150.0, 700.0)
    from open_source_einstar_b200 import SgmParams, StereoParams
    for ci, (r, s, w, h, pr) in enumerate(cal[:3]):  # every (size, D) kind, all slots, before the clock starts
        for d in SERVE_D:
            srv.reserve(w, h, StereoParams(sgm=SgmParams(min_disparity=pr.min_disparity, num_disparities=d)), ci,
                        slots)
    replay(srv, reqs, poisson_arrivals(480.0, 0.5, seed=99))  # warm-up
    clk = ClockSampler(dev.index or 0).__enter__()
    results = []
    for k, rate in enumerate(rates):
        arr = poisson_arrivals(rate, duration, seed=100 + k)
        comps, wall = replay(srv, reqs, arr)
        bad = [c for c in comps if not c.ok]
        if bad:
            raise SystemExit(f"{len(bad)} frames failed (status {bad[0].status})")
        lat = [c.latency_ms for c in comps]
        pxd = sum(reqs[c.tag % len(reqs)]["px_d"] for c in comps)
        summ = latency_summary(lat, wall)
        summ.update({"rate_hz": rate, "seconds": duration, "gpix_disp_per_s": pxd / wall / 1e9,
                     "gpu_ms_p50": float(np.percentile([c.gpu_ms for c in comps], 50)),
                     "queue_ms_p99": float(np.percentile([c.queue_ms for c in comps], 99))})
        results.append(summ)
    clk.__exit__(None, None, None)
    st = srv.stats()
    srv.close()
    line = {"metric": "serving frame latency p50/p99/p99.9 (ms) beside frames/s, Poisson arrivals",
            "workload": "serving", "unit": "ms", "higher_is_better": False, "n_gpus": world,
            "value": max(r["p99_ms"] for r in results), "value_is": "worst p99 latency over the rates",
            "rates": results, "dtype": "u8", "data": "synthetic",
            "config": {"workload": "Poisson arrivals; sizes 70 % 1280x1024, 20 % 960x768, 10 % 640x512 (raw pairs, "
                                   "GPU remap); D in {96, 128}; 4 resident synthetic rigs x 3 sizes; 40 GB volume "
                                   "budget; latency = submit -> u16 disparity + depth in pinned host memory",
                       "slots": slots, "parallelism": f"replicas x{world}"},
            "server": {"peak_running": st["peak_running"], "slots": st["slots"],
                       "volume_bytes": st["volume_bytes"], "device_bytes": st["device_bytes"]},
            "clocks": clk.summary()}
    return line


# ---- uneven batch: 64 rectified pairs of three sizes and four disparity ranges in one graph replay -----------
def run_batch64(args, world, rank, local):
    """64 pairs (24 x 640x512, 24 x 1280x1024, 16 x 960x768; D from {64, 96, 128, 192}; each its own
    calibration) as one StereoBatch graph replay with autotuned kernels and schedule, against the same
    pairs launched per frame (one handle per pair, back to back on one stream). Bit-exact check first."""
    import torch
    torch.cuda.set_device(local)
    line = batch64_line(torch.device("cuda", local), args.steps, args.warmup, world, rank, tune_schedule=True)
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def batch64_line(dev, steps, warmup, world=1, rank=0, tune_schedule=True):
    """The 64-pair uneven batch's JSON line (configuration 3) on device `dev`; without tune_schedule the
    library's default (micro_batch, branches) is used."""
    import torch
    from open_source_einstar_b200 import (CudaStereo, PairDesc, RectifiedGeometry, SgmParams, StereoBatch, StereoParams,
                                          synth)
    from open_source_einstar_b200.autotune import Autotuner, FrameKind, tune_batch_schedule
    pairs = synth.batch_pairs(64, seed=rank, device=dev)
    tuner = Autotuner()
    descs, handles, ins, outs = [], [], [], []
    for pr in pairs:
        h, w = pr.left.shape
        sp = StereoParams(sgm=SgmParams(min_disparity=pr.min_disparity, num_disparities=pr.num_disparities))
        kcfg = tuner.tune(FrameKind.of(w, h, sp))              # per-frame path
        bcfg = tuner.tune(FrameKind.of(w, h, sp), batch=True)  # batched path
        geom = RectifiedGeometry(pr.f, 0, 0, pr.baseline, 0.0)
        descs.append(PairDesc(w, h, sp, geometry=geom, kernel=bcfg))
        s = CudaStereo.create(sp, w, h)
        from open_source_einstar_b200.autotune import apply
        apply(s, kcfg)
        s.set_point_params(geom, 150.0, 700.0)
        handles.append(s)
        ins.append((torch.from_numpy(pr.left).to(dev), torch.from_numpy(pr.right).to(dev)))
        outs.append({"disparity_u16": torch.empty((h, w), dtype=torch.int16, device=dev),
                     "depth": torch.empty((h, w), dtype=torch.float32, device=dev)})
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    px_d = sum(p.left.shape[0] * p.left.shape[1] * p.num_disparities for p in pairs)
    formula = sum(algorithmic_bytes(p.left.shape[1], p.left.shape[0], p.num_disparities, P, raw=False) for p in pairs)

    def per_frame():
        for s, (l, r), o in zip(handles, ins, outs):
            s.compute_device(l, r, o, stream=stream)

    def make_batch(mb, br):
        b = StereoBatch(descs, micro_batch=mb, branches=br)
        for i, ((l, r), o) in enumerate(zip(ins, bouts)):
            b.bind(i, l, r, o)
        return b

    def time_run(b):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.run(stream=stream)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    bouts = [{k: torch.empty_like(v) for k, v in o.items()} for o in outs]
    if tune_schedule:
        (mb, br), sched = tune_batch_schedule(make_batch, time_run, len(descs))
    else:
        mb, br, sched = 0, 0, {}
    batch = make_batch(mb, br)
    mb, br = batch.micro_batch, batch.branches
    for _ in range(warmup):
        per_frame()
        batch.run(stream=stream)
    torch.cuda.synchronize(dev)
    for i, (o, bo) in enumerate(zip(outs, bouts)):
        if not (torch.equal(o["disparity_u16"], bo["disparity_u16"]) and torch.equal(o["depth"], bo["depth"])):
            raise SystemExit(f"pair {i}: batched and per-pair outputs differ")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk = ClockSampler(dev.index or 0).__enter__()
    e0.record(stream)
    for _ in range(steps):
        per_frame()
    e1.record(stream)
    e1.synchronize()
    pf_ms = e0.elapsed_time(e1) / steps
    e0.record(stream)
    for _ in range(steps):
        batch.run(stream=stream)
    e1.record(stream)
    e1.synchronize()
    b_ms = e0.elapsed_time(e1) / steps
    clk.__exit__(None, None, None)
    hbm, hbm_kind = peaks()
    line = {"metric": "batched SGM Gpix*disp/s, 64 uneven pairs in one graph replay vs per-frame launches",
            "workload": "batch64", "value": px_d / (b_ms * 1e-3) / 1e9, "unit": UNIT, "higher_is_better": True,
            "n_gpus": world, "steps": steps, "warmup": warmup, "ms_per_step": b_ms,
            "per_frame": {"value": px_d / (pf_ms * 1e-3) / 1e9, "ms_per_step": pf_ms},
            "batched_over_per_frame": pf_ms / b_ms,
            "pipeline_frac": formula / (b_ms * 1e-3) / 1e9 / hbm, "peak_gbs": hbm, "peak_kind": hbm_kind,
            "pipeline_formula_bytes": formula,
            "schedule": {"micro_batch": mb, "branches": br,
                         "tried_ms": {f"{k[0]}x{k[1]}": v for k, v in sorted(sched.items())}},
            "launches_per_run": batch.launches_per_run, "device_bytes": batch.device_bytes,
            "kernels": sorted({json.dumps(d.kernel, sort_keys=True) for d in descs}),
            "dtype": "u8", "data": "synthetic",
            "config": {"workload": "24 x 640x512, 24 x 1280x1024, 16 x 960x768 rectified plane+sphere speckle pairs, "
                                   "D from {64, 96, 128, 192}, f 800-1200 px, baseline 50-70 mm; 4-path SGM, WTA, "
                                   "L-R, median, u16 + depth", "parallelism": f"replicas x{world}"},
            "clocks": clk.summary()}
    batch.close()
    for s in handles:
        s.close()
    torch.cuda.set_stream(torch.cuda.default_stream(dev))
    return line


# ---- offline re-depth: a raw recording in batches of 128 at D=256, 8 paths, u16 path values -----------------
def run_offline(args, world, rank, local):
    """Configuration 5 on its own line (see offline_line)."""
    import torch
    torch.cuda.set_device(local)
    line = offline_line(torch.device("cuda", local), args.recording_frames, args.offline_batch, world, rank, local)
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def offline_line(dev, n, batch, world=1, rank=0, local=0):
    """A synthetic handheld recording (150 mm object, 250-450 mm standoff, raw 1280x1024 IR pairs) of `n`
    frames re-depthed in batches of `batch` frames: 8-path SGM, D=256, 16-bit path values. Frames are
    rendered into pinned host memory first (untimed); the timed run covers host->device copies, the batched
    graph replays and device->host copies of u16 disparity and depth, double-buffered. Three frames are
    checked against the per-frame path first. Returns the JSON line (configuration 5)."""
    from open_source_einstar_b200 import CudaStereo, RectifiedGeometry, RemapTable, SgmParams, StereoParams, synth
    from open_source_einstar_b200.autotune import Autotuner, FrameKind
    from open_source_einstar_b200.offline import OfflineRedepth
    from open_source_einstar_b200.serving import pinned_empty
    W_, H_, D_ = 1280, 1024, 256
    rec = synth.recording(n_frames=n, seed=rank, width=W_, height=H_, num_disparities=D_, device=dev)
    lefts, rights = pinned_empty((n, H_, W_), np.uint8), pinned_empty((n, H_, W_), np.uint8)
    for i in range(n):
        lefts[i], rights[i] = synth.recording_frame(rec, i, device=dev)
    sp = StereoParams(sgm=SgmParams(min_disparity=rec.min_disparity, num_disparities=D_, eight_paths=True),
                      wide_costs=True)
    geom = RectifiedGeometry(rec.rect.f, 0, 0, rec.rect.baseline, rec.rect.cx_offset)
    kernel = Autotuner().tune(FrameKind.of(W_, H_, sp), batch=True)
    out_u16 = pinned_empty((n, H_, W_), np.uint16)
    out_depth = pinned_empty((n, H_, W_), np.float32)
    with OfflineRedepth(W_, H_, sp, rec.maps, (W_, H_), geom, batch_size=batch, kernel=kernel) as off:
        warm = min(n, 2 * batch)
        off.run(lefts[:warm], rights[:warm], out_u16[:warm], out_depth[:warm])
        clk = ClockSampler(local).__enter__()
        st = off.run(lefts, rights, out_u16, out_depth)
        clk.__exit__(None, None, None)
        dev_bytes = off.device_bytes
    # spot check: frames re-depthed alone through the per-frame path are identical
    (lx, ly), (rx, ry) = rec.maps
    with CudaStereo.create(sp, W_, H_) as s:
        s.set_rectification(RemapTable(lx, ly), RemapTable(rx, ry), W_, H_)
        s.set_point_params(geom, 150.0, 700.0)
        for i in (0, n // 2, n - 1):
            r = s.compute_raw(lefts[i], rights[i])
            if not (np.array_equal(r.disparity_u16, out_u16[i]) and np.array_equal(r.depth.view(np.uint32),
                                                                                   out_depth[i].view(np.uint32))):
                raise SystemExit(f"offline frame {i} differs from the per-frame path")
    hbm, hbm_kind = peaks()
    ms = st.device_ms
    formula = algorithmic_bytes(W_, H_, D_, 8, c_b=2, raw=True) * n
    line = {"metric": f"offline re-depth Gpix*disp/s, 8-path D=256 u16, batches of {batch} raw 1280x1024 frames",
            "workload": "offline", "value": n * W_ * H_ * D_ / (ms * 1e-3) / 1e9, "unit": UNIT,
            "higher_is_better": True, "n_gpus": world, "frames": n, "batches": st.batches,
            "frames_per_s": n / (ms * 1e-3), "ms_per_frame": ms / n,
            "pipeline_frac": formula / (ms * 1e-3) / 1e9 / hbm, "pipeline_formula_bytes_per_frame": formula // n,
            "peak_gbs": hbm, "peak_kind": hbm_kind, "device_bytes": dev_bytes, "kernel": kernel,
            "dtype": "u16", "data": "synthetic",
            "config": {"workload": f"synthetic handheld recording of {n} raw 1280x1024 IR pairs (12-primitive 150 mm "
                                   "object on a base plane, 250-450 mm standoff, speckle, sigma 2 DN); GPU remap, "
                                   "8-path SGM D=256 with u16 path values, WTA, L-R, median, u16 + depth; "
                                   "timed: H2D + batched graph replays + D2H, double-buffered",
                       "batch": batch, "parallelism": f"replicas x{world}"},
            "clocks": clk.summary()}
    return line


def frontend_params(f, baseline):
    """The scanner frontend's depth::StereoParams (stereo_frontend.cpp:21-34): stereo on the half-resolution
    rectified pair, SGM a level below over the quarter-resolution disparities of 150-700 mm (+/- 2 px
    guard), the reference's refinement, detail, filter and speckle defaults."""
    import math
    from open_source_einstar_b200 import SgmParams, StereoParams
    fq = f / 4.0
    d_max, d_min = fq * baseline / 150.0, fq * baseline / 700.0
    sgm = SgmParams(min_disparity=int(math.floor(d_min)) - 2, num_disparities=int(math.ceil(d_max - d_min)) + 4)
    return StereoParams(pyramid_levels=1, sgm=sgm, median=False, detail_enabled=True, filter_occlusion=True,
                        filter_spikes=True, speckle_max_region_size=200)


def reference_frontend_frame(ref, pair, sp):
    """The CPU frontend's depth step on one raw pair (stereo_frontend.cpp:331-335): remap both images at
    full resolution, box-downsample, depth::compute_disparity with the full-resolution pair (oracle/_ref)."""
    (lx, ly), (rx, ry) = pair.maps
    t0 = time.perf_counter()
    fl, fr = ref.remap(pair.left, lx, ly), ref.remap(pair.right, rx, ry)
    d, c = ref.compute_disparity(ref.downsample2(fl), ref.downsample2(fr), sp, fl, fr)
    return time.perf_counter() - t0, d, c


def run_frontend(args, world, rank, local):
    """The scanner frontend's whole depth step (depth::compute_disparity as stereo_frontend.cpp configures
    it) on raw 1280x1024 pairs: full-resolution GPU remap, box downsample to 640x512, SGM at 320x256,
    slanted ZNCC refinement to 640x512, detail refinement on the 1280x1024 pair, occlusion and spike
    filters, speckle removal. One step = --frames frames; metric frames/s."""
    import torch
    from open_source_einstar_b200 import CudaStereo, RemapTable
    from open_source_einstar_b200.stereo import STAGE_NAMES, kernel_launches
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    B = args.frames
    pairs = make_frames(B, replica_seed0(rank), dev)
    (lx, ly), (rx, ry) = pairs[0].maps
    sp = frontend_params(pairs[0].f, pairs[0].baseline)
    w, h = W // 2, H // 2
    s = CudaStereo.create(sp, w, h)
    s.set_rectification(RemapTable(lx, ly), RemapTable(rx, ry), W, H)
    raw = [(torch.from_numpy(p.left).to(dev), torch.from_numpy(p.right).to(dev)) for p in pairs]
    outs = [{"disparity": torch.empty((h, w), dtype=torch.float32, device=dev),
             "confidence": torch.empty((h, w), dtype=torch.float32, device=dev)} for _ in range(B)]
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)

    def step():
        for (l, r), o in zip(raw, outs):
            s.compute_device(l, r, o, stream=stream, raw=True)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    # the device results equal the host API's (which the parity tests hold to the reference)
    r0 = s.compute_raw(pairs[0].left, pairs[0].right)
    if not np.array_equal(r0.disparity.view(np.uint32), outs[0]["disparity"].cpu().numpy().view(np.uint32)):
        raise SystemExit("device-resident and host frames differ")
    clk = ClockSampler(local).__enter__()
    s.profile(True)
    s.profile_collect()
    l0 = kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    launches = kernel_launches() - l0
    ms = e0.elapsed_time(e1)
    stages = s.profile_collect(max_frames=B * args.steps + 8)
    s.profile(False)
    n_frames = B * args.steps
    # end to end through the host API: raw pair in from host memory, disparity + confidence back
    host = [(np.ascontiguousarray(p.left), np.ascontiguousarray(p.right)) for p in pairs]
    res = [s.compute_raw(*host[0])]
    t0 = time.perf_counter()
    for i in range(n_frames):
        res[0] = s.compute_raw(*host[i % B])
    e2e_s = time.perf_counter() - t0
    # the frontend's own per-frame call (ds_compute_frame): points, normals and weights left on the device,
    # marker blobs of both raw images (stickers composited into the scenes) handed over during the stereo
    from open_source_einstar_b200 import BlobParams, RectifiedGeometry, synth
    s.set_point_params(RectifiedGeometry(pairs[0].f / 2, (w - 1) / 2.0, (h - 1) / 2.0, pairs[0].baseline, 0.0), 150.0, 700.0, 4.0)
    s.set_blob_params(BlobParams())
    marked = [(synth.add_markers((p.left * 0.6).astype(np.uint8), n_markers=20, seed=2 * k)[0],
               synth.add_markers((p.right * 0.6).astype(np.uint8), n_markers=20, seed=2 * k + 1)[0]) for k, p in enumerate(pairs[:2])]
    pts = torch.empty((h, w, 4), dtype=torch.float32, device=dev)
    nrm = torch.empty((h, w, 4), dtype=torch.float32, device=dev)
    wts = torch.empty((h, w), dtype=torch.float32, device=dev)
    fr = s.compute_frame(*marked[0], pts, nrm, wts, blobs=True)
    t0 = time.perf_counter()
    for i in range(n_frames):
        fr = s.compute_frame(*marked[i % 2], pts, nrm, wts, blobs=True)
    frame_s = time.perf_counter() - t0
    blob_counts = [len(fr.blobs[0]), len(fr.blobs[1])]
    clk.__exit__(None, None, None)
    s.close()
    frame_tot = stages.sum(axis=1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle.oracle import Ref
        ref = Ref()
        cpu_pairs = make_frames(2, 0, dev)
        reference_frontend_frame(ref, cpu_pairs[0], sp)
        times = []
        t_start = time.perf_counter()
        while len(times) < 8 and time.perf_counter() - t_start < 20.0:
            times.append(reference_frontend_frame(ref, cpu_pairs[len(times) % 2], sp)[0])
        med = statistics.median(times)
        cpu = {"value": 1e3 / (med * 1e3), "unit": "frames/s", "cores": ref.threads(), "kind": "reference",
               "ms_per_frame": med * 1e3,
               "sample": f"{len(times)} raw 1280x1024 frames: restated calib::remap x2, the reference's downsample2 and "
                         "compute_disparity (oracle/_ref: libs/depth/src/stereo.cpp) over "
                         f"{ref.threads()} threads"}
    if rank == 0:
        line = {"metric": "frontend depth frames/s (depth::compute_disparity as the scanner frontend runs it), raw 1280x1024",
                "workload": "frontend", "value": n_frames / (ms * 1e-3), "unit": "frames/s", "higher_is_better": True,
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "ms_per_frame": ms / n_frames, "dtype": "u8/f32/f64", "data": "synthetic", "vs_baseline": None,
                "scaling": "weak",
                "frame_ms": {"p50": float(np.percentile(frame_tot, 50)), "p99": float(np.percentile(frame_tot, 99))},
                "stage_ms": {"rectify_downsample": float(stages[:, 0].mean()),
                             "sgm_320x256": float(stages[:, 1:5].sum(axis=1).mean()),
                             "refine_detail_filters_speckles": float(stages[:, 5].mean())},
                "config": {"workload": "raw 1280x1024 u8 pairs (config-2 scenes): GPU remap at 1280x1024, 2x2 box to 640x512, "
                                       f"SGM 4 paths at 320x256 D={sp.sgm.num_disparities}, ZNCC refinement (7x7 slanted, "
                                       "+/-2 px in 0.5 px) to 640x512, detail refinement (10x10 at 1280x1024), occlusion + "
                                       "spike filters, speckles < 200 px removed",
                           "frames_per_step": B, "parallelism": f"replicas x{world}"},
                "e2e": {"value": n_frames / e2e_s, "unit": "frames/s", "h2d_bytes_per_step": B * 2 * W * H,
                        "d2h_bytes_per_step": B * w * h * 8,
                        "api": "CudaStereo.compute_raw (ds_compute_raw): host raw pair in, host disparity + confidence out, "
                               "wall clock"},
                "e2e_frame": {"value": n_frames / frame_s, "unit": "frames/s", "h2d_bytes_per_step": B * 2 * W * H,
                              "d2h_bytes_per_step": B * w * h * 10,
                              "api": "CudaStereo.compute_frame (ds_compute_frame): host raw pair in; points, normals, weights "
                                     "left on the device; disparity, confidence, u16 and the marker candidates of both raw "
                                     "images (20 stickers each) back on the host; wall clock",
                              "marker_candidates": blob_counts},
                "cpu_baseline": cpu, "gpu_launches": int(launches), "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    return 0


def plugin_leg(stereo, pairs, calls, warmup=3):
    """End to end through the drop-in call, one frame per call as the scanner frontend makes it
    (StereoFrontend::process -> compute_raw, stereo_frontend.cpp:317): CudaStereo.compute_raw, i.e.
    ds_compute_raw, with the raw pair in pinned host memory and the u16 disparity + depth written back to
    pinned host memory; the call returns when they are there. Host-clock latency per call and throughput."""
    from open_source_einstar_b200 import StereoResult
    from open_source_einstar_b200.serving import pinned_copy, pinned_empty
    host = [(pinned_copy(p.left), pinned_copy(p.right)) for p in pairs[:4]]
    res = StereoResult(disparity=None, confidence=None, disparity_u16=pinned_empty((H, W), np.uint16),
                       depth=pinned_empty((H, W), np.float32))
    for i in range(warmup):
        stereo.compute_raw(*host[i % len(host)], out=res)
    lat = []
    t0 = time.perf_counter()
    for i in range(calls):
        t = time.perf_counter()
        stereo.compute_raw(*host[i % len(host)], out=res)
        lat.append((time.perf_counter() - t) * 1e3)
    total = time.perf_counter() - t0
    return {"value": calls * PX_D / total / 1e9, "unit": UNIT, "calls": calls,
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "max": float(max(lat))},
            "h2d_bytes_per_call": 2 * W * H, "d2h_bytes_per_call": W * H * (2 + 4),
            "api": "CudaStereo.compute_raw (ds_compute_raw): raw pair from pinned host memory in, u16 disparity + f32 "
                   "depth in pinned host memory out, one frame per synchronous call; host clock"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames", type=int, default=16, help="frames per step (the batch)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--reference-budget", type=float, default=150.0, help="seconds of timed reference work at most")
    ap.add_argument("--kernel-config", default="", help="R,SEG,MATERIALIZE override (default: the library's choice)")
    ap.add_argument("--workload", default="frames", choices=["frames", "serving", "batch64", "offline", "frontend"],
                    help="frames: the 1280x1024 D=128 throughput line (default); serving: the request-server latency run")
    ap.add_argument("--duration", type=float, default=20.0, help="serving: seconds of arrivals per rate")
    ap.add_argument("--rates", type=float, nargs="+", default=[120.0, 240.0, 480.0], help="serving: arrival rates (Hz)")
    ap.add_argument("--slots", type=int, default=6, help="serving: frames on the GPU at once")
    ap.add_argument("--recording-frames", type=int, default=256, help="offline: frames of the synthetic recording")
    ap.add_argument("--offline-batch", type=int, default=128, help="offline: frames per batch")
    ap.add_argument("--no-extras", action="store_true",
                    help="default line without the serving and 64-pair batch summaries (single-GPU runs carry them)")
    ap.add_argument("--extras-duration", type=float, default=3.0, help="serving summary: seconds of arrivals per rate")
    ap.add_argument("--extras-offline-frames", type=int, default=64,
                    help="offline summary on the default line: frames of the synthetic recording (two batches)")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        return run_reference(args, world, rank)
    if args.workload == "serving":
        return run_serving(args, world, rank, local)
    if args.workload == "batch64":
        return run_batch64(args, world, rank, local)
    if args.workload == "offline":
        return run_offline(args, world, rank, local)
    if args.workload == "frontend":
        return run_frontend(args, world, rank, local)

    import torch
    from open_source_einstar_b200 import (CudaStereo, PairDesc, RectifiedGeometry, RemapTable, SgmParams, StereoBatch,
                                          StereoParams)
    from open_source_einstar_b200.batch import BATCH_STAGE_NAMES
    from open_source_einstar_b200.stereo import STAGE_NAMES, kernel_launches

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    B = args.frames
    pairs = make_frames(B, replica_seed0(rank), dev)
    (lx, ly), (rx, ry) = pairs[0].maps
    sp = StereoParams(sgm=SgmParams(min_disparity=pairs[0].min_disparity, num_disparities=D))
    geom = RectifiedGeometry(pairs[0].f, 0, 0, pairs[0].baseline, 0.0)
    kcfg = None
    if args.kernel_config:
        r, seg, mat = (int(v) for v in args.kernel_config.split(","))
        kcfg = {"regs_per_lane": r, "lanes_per_line": seg, "materialize_costs": mat, "prefetch_steps": 8}
    raw = [(torch.from_numpy(p.left).to(dev), torch.from_numpy(p.right).to(dev)) for p in pairs]
    outs = [{"disparity_u16": torch.empty((H, W), dtype=torch.int16, device=dev),
             "depth": torch.empty((H, W), dtype=torch.float32, device=dev)} for _ in range(B)]
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(dev)

    def job_max(v: float) -> float:
        return max_over_ranks(v, world, dev)

    clk = ClockSampler(local).__enter__()

    # ---- per-frame launch path: one handle, frames back to back on one stream ----------------------------
    s = CudaStereo.create(sp, W, H)
    s.set_rectification(RemapTable(lx, ly), RemapTable(rx, ry), W, H)
    s.set_point_params(geom, 150.0, 700.0)
    if kcfg:
        s.set_kernel_config(kcfg["regs_per_lane"], kcfg["lanes_per_line"], bool(kcfg["materialize_costs"]), 4, 256, 8)

    def frame_step():
        for (l, r), o in zip(raw, outs):
            s.compute_device(l, r, o, stream=stream, raw=True)

    for _ in range(args.warmup):
        frame_step()
    barrier()
    s.profile(True)
    s.profile_collect()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    for _ in range(args.steps):
        frame_step()
    e1.record(stream)
    barrier()
    pf_ms = job_max(e0.elapsed_time(e1))
    stages = s.profile_collect(max_frames=B * args.steps + 8)
    s.profile(False)
    frame_tot = stages.sum(axis=1) if len(stages) else np.zeros(1)
    per_frame_value = B * args.steps * world * PX_D / (pf_ms * 1e-3) / 1e9

    # ---- batched path: all frames in one graph replay (persistent launches) -----------------------------
    desc = [PairDesc(W, H, sp, raw=True, calib=0, geometry=geom, kernel=kcfg) for _ in range(B)]
    batch = StereoBatch(desc, n_calib=1)
    batch.set_rectification(0, RemapTable(lx, ly), RemapTable(rx, ry), W, H)
    bouts = [{"disparity_u16": torch.empty((H, W), dtype=torch.int16, device=dev),
              "depth": torch.empty((H, W), dtype=torch.float32, device=dev)} for _ in range(B)]
    for i, ((l, r), o) in enumerate(zip(raw, bouts)):
        batch.bind(i, l, r, o)
    batch.profile(True)
    for _ in range(args.warmup):
        batch.run(stream=stream)
    barrier()
    for o, bo in zip(outs, bouts):  # the batched results equal the per-frame ones
        if not (torch.equal(o["disparity_u16"], bo["disparity_u16"]) and torch.equal(o["depth"], bo["depth"])):
            raise SystemExit("batched and per-frame outputs differ")
    launches0 = kernel_launches()
    barrier()
    e0.record(stream)
    for _ in range(args.steps):
        batch.run(stream=stream)
    e1.record(stream)
    barrier()
    launches = batch.launches_per_run * args.steps  # graph replays launch the captured kernels
    ms = job_max(e0.elapsed_time(e1))
    bstage = batch.stage_ms()
    frames_total = B * args.steps * world
    value = frames_total * PX_D / (ms * 1e-3) / 1e9

    # ---- end to end through the public API (OfflineRedepth over StereoBatch): every step copies its 16 raw
    # pairs in from pinned host memory and its u16 disparities and depths out to pinned host memory. Steps
    # are double-buffered, so one step's copies overlap another's compute; the time runs on the device from
    # the first copy in to the last copy out.
    from open_source_einstar_b200.offline import OfflineRedepth
    from open_source_einstar_b200.serving import pinned_empty
    e2e_steps = max(2, args.steps)  # the K steps of the device-timed region, through the host API
    n_e2e = B * e2e_steps
    host_l, host_r = pinned_empty((B, H, W), np.uint8), pinned_empty((B, H, W), np.uint8)
    for i, p in enumerate(pairs):
        host_l[i], host_r[i] = p.left, p.right
    ring_u16, ring_depth = pinned_empty((2 * B, H, W), np.uint16), pinned_empty((2 * B, H, W), np.float32)
    e2e_l = [host_l[i % B] for i in range(n_e2e)]
    e2e_r = [host_r[i % B] for i in range(n_e2e)]
    e2e_u16 = [ring_u16[i % (2 * B)] for i in range(n_e2e)]
    e2e_depth = [ring_depth[i % (2 * B)] for i in range(n_e2e)]
    off = OfflineRedepth(W, H, sp, pairs[0].maps, (W, H), geom, batch_size=B, kernel=kcfg)
    off.run(e2e_l[:2 * B], e2e_r[:2 * B], e2e_u16[:2 * B], e2e_depth[:2 * B])  # warm-up (graph capture)
    barrier()
    est = off.run(e2e_l, e2e_r, e2e_u16, e2e_depth)
    e2e_s = job_max(est.device_ms) * 1e-3
    e2e_value = n_e2e * world * PX_D / e2e_s / 1e9
    for j in range(B):  # the last step's results, copied out, equal the per-frame path's
        if not np.array_equal(e2e_u16[n_e2e - B + j], outs[j]["disparity_u16"].cpu().numpy().view(np.uint16)):
            raise SystemExit("end-to-end outputs differ from the per-frame path")
    off.close()
    plug = plugin_leg(s, pairs, max(16, 2 * args.steps))
    clk.__exit__(None, None, None)

    # ---- roofline of the dominant kernel: the SGM path launch (k_paths), one frame per launch, timed by the
    # stage events around it on the stream it runs on during the per-frame timed region (frames back to back,
    # nothing else on the GPU). The batched path runs the same kernel body as persistent launches (kb_paths)
    # on concurrent graph branches; its branch-0 launch time is reported beside it.
    hbm, hbm_kind = peaks()
    path_bytes = path_stage_bytes(W, H, D, P)
    stage_mean = stages.mean(axis=0) if len(stages) else np.zeros(len(STAGE_NAMES))
    paths_ms = float(stage_mean[STAGE_NAMES.index("paths")])
    achieved = path_bytes / (paths_ms * 1e-3) / 1e9 if paths_ms > 0 else 0.0
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "paths_traffic.json")) as f:
            traffic = json.load(f).get("k_paths", {}).get("dram_bytes_per_launch")
    except Exception:
        pass
    bpaths_ms = float(bstage[BATCH_STAGE_NAMES.index("paths")])
    micro = batch.micro_batch
    roofline = {"bound": "hbm", "kernel": "k_paths (SGM path aggregation, 4 directions, one frame per launch)",
                "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "peak_kind": f"{hbm_kind} hbm_gbs (burst copy; the kernel is timed alone)",
                "traffic": traffic, "algorithmic_bytes_per_launch": path_bytes, "kernel_ms": paths_ms,
                "share_of_frame": paths_ms / max(float(stage_mean.sum()), 1e-9),
                "batched": {"kernel": "kb_paths", "frames_per_launch": micro, "concurrent_branches": batch.branches,
                            "kernel_ms_branch0": bpaths_ms,
                            "achieved_per_launch_gbs": path_bytes * micro / (bpaths_ms * 1e-3) / 1e9 if bpaths_ms > 0 else 0.0,
                            "stage_ms_branch0": {n: float(v) for n, v in zip(BATCH_STAGE_NAMES, bstage)}},
                "pipeline_formula_bytes_per_frame": algorithmic_bytes(W, H, D, P),
                "pipeline_frac": algorithmic_bytes(W, H, D, P) * B / (ms / args.steps * 1e-3) / 1e9 / hbm}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from open_source_einstar_b200 import synth
        cpu_pairs = [synth.raw_objects_pair(seed=i, device=dev) for i in range(2)]
        cpu = cpu_reference_sample(cpu_pairs)

    h2d = B * 2 * W * H
    d2h = B * W * H * (2 + 4)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": WORKLOAD, "frames_per_step": B,
                       "path": "batched: persistent launches per stage over all frames, one CUDA graph replay per step",
                       "kernel_config": s.kernel_config(),
                       "l2": "working set per frame (~0.84 GB of cost and path volumes) far above the 126 MB L2",
                       "parallelism": f"replicas x{world}"},
            "per_frame": {"value": per_frame_value, "unit": UNIT, "ms_per_frame": pf_ms / (args.steps * B),
                          "frame_ms": {"p50": float(np.percentile(frame_tot, 50)), "p99": float(np.percentile(frame_tot, 99))},
                          "stage_ms": {n: float(v) for n, v in zip(STAGE_NAMES, stages.mean(axis=0))} if len(stages) else {}},
            "batched_over_per_frame": value / per_frame_value,
            "frame_ms": {"p50": float(np.percentile(frame_tot, 50)), "p99": float(np.percentile(frame_tot, 99)),
                         "batch_latency_ms": ms / args.steps},
            "roofline": roofline, "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "api": "OfflineRedepth (StereoBatch graph replays, ds_batch_run) with every step's raw pairs copied in "
                           "from pinned host memory and its u16 disparity + depth copied out; steps double-buffered",
                    "steps": e2e_steps},
            "e2e_plugin": plug,
            "gpu_launches": int(launches), "clocks": clk.summary()}
    batch.close()
    s.close()
    if world == 1 and not args.no_extras:
        # configurations 4, 3 and 5 on the same box: the request server under Poisson arrivals (a shorter run per
        # rate than --workload serving), the 64-pair uneven batch against per-frame launches, and a 64-frame
        # offline re-depth (8 paths, D=256, u16 path values; --workload offline runs the longer recording)
        srv = serving_line(dev, args.rates, args.extras_duration, args.slots)
        line["serving"] = {"rates": srv["rates"], "worst_p99_ms": srv["value"], "slots": srv["config"]["slots"],
                           "seconds_per_rate": args.extras_duration, "clocks": srv["clocks"]}
        b64 = batch64_line(dev, 3, 2, tune_schedule=False)
        line["batch64"] = {k: b64[k] for k in ("value", "unit", "ms_per_step", "per_frame", "batched_over_per_frame",
                                               "pipeline_frac", "schedule", "launches_per_run", "kernels", "clocks")}
        line["batch64"]["bit_exact_vs_per_frame"] = True  # batch64_line stops the run otherwise
        off = offline_line(dev, args.extras_offline_frames, args.extras_offline_frames // 2, world, rank, local)
        line["offline"] = {k: off[k] for k in ("value", "unit", "frames", "batches", "frames_per_s", "ms_per_frame",
                                               "pipeline_frac", "peak_kind", "kernel", "clocks")}
        line["offline"]["spot_checked_vs_per_frame"] = True  # offline_line stops the run otherwise
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
