"""Kernel-configuration autotuner for the SGM kernels (ds_set_kernel_config / PairDesc.kernel).

For one kind of frame (width, height, disparities, paths, value width, census window) it times candidate
kernel configurations on the device and keeps the fastest one. Results are cached in a JSON table keyed
by the frame kind and the GPU name. Every configuration gives bit-identical results (the parity tests
hold each one to the oracle), so tuning changes speed only.

The knobs (ds_kernel_config in include/depth_cuda.h):
- lanes_per_line (SEG) x regs_per_lane (R): the tile shape of a scanline. SEG lanes each hold a
  disparity slab 2R deep, and SEG*2R >= D. SEG 16 puts two scanlines in a warp.
- path_warps_per_block: paths per block. The block holds path_warps * 32/SEG scanlines, which are
  neighbours in the image, so the vertical and diagonal directions read adjacent cache lines.
- materialize_costs: write the cost volume once and read it per direction, or recompute each cost
  from the census words in every direction.
- prefetch_steps: steps of cost / census input kept in flight per scanline (4 or 8).
- wta_threads: threads per winner-takes-all block (the per-pixel WTA; frames that the row-sweep WTA runs,
  4 paths with byte values and a 48/64/96/128-disparity slab, skip this stage).
- fused_pairs (4 directions): the two sweep kernels instead of cost / path / WTA kernels: the vertical path
  pair, then the horizontal pair with the WTA and the L-R check. They need byte pair sums
  (2 (window + P2) <= 255), census windows of at most 32 neighbours and D <= 128, with 4 or 8 lanes per
  line of 12 or 16 disparities; their block shapes are fixed.

The search is staged: tile shape x materialisation (and the sweep shapes), then paths per block x
prefetch, then the WTA block. That is about 16 timed configurations instead of the full product. The
per-frame path and the batched path are tuned separately (a batch keeps many frames in flight, so its
best kernels can differ).

    python -m open_source_einstar_b200.autotune 1280x1024:128 640x512:64 --batch --write
"""
from __future__ import annotations

import argparse
import json
import os
import time
from dataclasses import dataclass

import numpy as np

PACKAGE_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning", "b200.json")
SUPPORTED = {8: (4, 6, 8), 16: (1, 2, 3, 4), 32: (1, 2, 3, 4, 6, 8)}
SWEEP_SHAPES = {4: (6, 8), 8: (6, 8)}  # lanes per line -> registers per lane of the sweep kernels
DEFAULT = {"path_warps_per_block": 4, "wta_threads": 256, "prefetch_steps": 8, "fused_pairs": 0,
           "horz_warps_per_block": 4}


@dataclass(frozen=True)
class FrameKind:
    width: int
    height: int
    num_disparities: int
    eight_paths: bool = False
    wide: bool = False          # u16 path values (window + P2 > 255 or forced)
    census_window: int = 25
    byte_pair_sums: bool = True  # 2 (window + P2) <= 255 (not part of the key: it follows from the parameters)

    def key(self, device: str) -> str:
        return (f"{device}|{self.width}x{self.height}|D{self.num_disparities}|P{8 if self.eight_paths else 4}|"
                f"{'u16' if self.wide else 'u8'}|w{self.census_window}")

    @staticmethod
    def of(width: int, height: int, params) -> "FrameKind":
        s = params.sgm
        window = (2 * s.census_radius_x + 1) * (2 * s.census_radius_y + 1)
        wide = bool(params.wide_costs or window + s.p2 > 255)
        return FrameKind(int(width), int(height), int(s.num_disparities), bool(s.eight_paths), wide, window,
                         not wide and 2 * (window + s.p2) <= 255)

    def row_wta_fit(self, dp: int) -> bool:
        """Whether the library runs the WTA of this kind of frame as row sweeps (k_wta_rows, wta_rows_fit):
        4 paths, byte pair sums and a lane slab of 48, 64, 96 or 128 disparities."""
        return not self.eight_paths and self.byte_pair_sums and dp in (48, 64, 96, 128)

    def sweep_fit(self) -> bool:
        """Whether the sweep kernels can run this kind of frame (the library's own check, sweep_unfit)."""
        return (not self.eight_paths and self.byte_pair_sums and self.census_window - 1 <= 32
                and self.num_disparities <= 128)


def tile_shapes(num_disparities: int) -> list[tuple[int, int]]:
    """(R, SEG) pairs with the fewest padded disparities for each SEG: SEG*2R >= D, R supported."""
    out = []
    for seg, rs in SUPPORTED.items():
        fit = [r for r in rs if seg * 2 * r >= num_disparities]
        if fit:
            out.append((min(fit), seg))
    return out


def sweep_shapes(num_disparities: int) -> list[tuple[int, int]]:
    """(R, SEG) of the sweep kernels with the fewest padded disparities for each SEG (SEG*2R >= D)."""
    out = []
    for seg, rs in SWEEP_SHAPES.items():
        fit = [r for r in rs if seg * 2 * r >= num_disparities]
        if fit:
            out.append((min(fit), seg))
    return out


def stage_candidates(kind: FrameKind, stage: int, best: dict | None = None, fused_ok: bool = True) -> list[dict]:
    """Candidates of one search stage (1: tile x materialisation, and the sweep shapes; 2: warps x prefetch;
    3: WTA). fused_ok=False leaves the sweep kernels out."""
    if stage == 1:
        c = []
        for r, seg in tile_shapes(kind.num_disparities):
            for mat in (1, 0):
                c.append({"regs_per_lane": r, "lanes_per_line": seg, "materialize_costs": mat, **DEFAULT})
        if fused_ok and kind.sweep_fit():
            for r, seg in sweep_shapes(kind.num_disparities):
                c.append({"regs_per_lane": r, "lanes_per_line": seg, "materialize_costs": 0, **DEFAULT, "fused_pairs": 1})
        return c
    assert best is not None
    if best.get("fused_pairs"):
        return [best]  # the sweep kernels have fixed block shapes
    if stage == 2:
        return [{**best, "path_warps_per_block": pw, "prefetch_steps": pf} for pw in (1, 2, 4, 8) for pf in (4, 8)]
    if kind.row_wta_fit(best["regs_per_lane"] * 2 * best["lanes_per_line"]):
        return [best]  # the row-sweep WTA runs these frames with a fixed block shape
    return [{**best, "wta_threads": t} for t in (128, 256)]


def search(kind: FrameKind, time_fn, fused_ok: bool = True, keep: int = 2) -> tuple[dict, dict]:
    """Staged search; time_fn(config) -> ms per frame (inf if the configuration is rejected). The `keep`
    fastest shapes of stage 1 each go through stage 2 (a shape's best block size can reorder them).
    Returns (best configuration, {stage: [(config, ms), ...]})."""
    log: dict = {}
    best, best_ms = None, float("inf")
    trials = [(cfg, time_fn(cfg)) for cfg in stage_candidates(kind, 1, None, fused_ok)]
    log[1] = trials
    finite = sorted((t for t in trials if t[1] != float("inf")), key=lambda t: t[1])
    if finite:
        best, best_ms = finite[0]
    seeds = [c for c, _ in finite[:keep]]
    log[2] = []
    for seed in seeds:
        for cfg in stage_candidates(kind, 2, seed, fused_ok):
            ms = time_fn(cfg)
            log[2].append((cfg, ms))
            if ms < best_ms:
                best, best_ms = cfg, ms
    log[3] = []
    if best is not None:
        for cfg in stage_candidates(kind, 3, best, fused_ok):
            ms = time_fn(cfg)
            log[3].append((cfg, ms))
            if ms < best_ms:
                best, best_ms = cfg, ms
    return best, {"ms": best_ms, "trials": log}


class Autotuner:
    """Tuned configurations by frame kind: the packaged B200 table, then a user table (read/written)."""

    def __init__(self, table_path: str | None = None, read_package_table: bool = True):
        self.table_path = table_path or os.environ.get("DS_TUNING_TABLE") or os.path.join(
            os.path.expanduser("~"), ".cache", "open_source_einstar_b200", "tuning.json")
        self.table: dict = {}
        if read_package_table and os.path.exists(PACKAGE_TABLE):
            with open(PACKAGE_TABLE) as f:
                self.table.update(json.load(f).get("entries", {}))
        if os.path.exists(self.table_path):
            with open(self.table_path) as f:
                self.table.update(json.load(f).get("entries", {}))

    @staticmethod
    def device_name() -> str:
        import torch
        return torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"

    @staticmethod
    def _key(kind: FrameKind, device: str, batch: bool) -> str:
        return kind.key(device) + ("|batch" if batch else "")  # the batched path is tuned separately

    def lookup(self, kind: FrameKind, device: str | None = None, batch: bool = False) -> dict | None:
        e = self.table.get(self._key(kind, device or self.device_name(), batch))
        return dict(e["config"]) if e else None

    def save(self, path: str | None = None) -> str:
        path = path or self.table_path
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        with open(path, "w") as f:
            json.dump({"format": 1, "entries": self.table}, f, indent=1, sort_keys=True)
        return path

    def tune(self, kind: FrameKind, frames: int = 8, warmup: int = 2, force: bool = False, batch: bool = False,
             params=None) -> dict:
        """The fastest configuration for `kind` on the per-frame path (batch=False) or the batched path,
        timed on the current GPU unless already in the table."""
        dev = self.device_name()
        if not force:
            hit = self.lookup(kind, dev, batch)
            if hit:
                return hit
        time_fn = batch_timer(kind, warmup, params) if batch else device_timer(kind, frames, warmup, params)
        best, info = search(kind, time_fn)
        self.table[self._key(kind, dev, batch)] = {
            "config": best, "ms_per_frame": info["ms"],
            "trials": [[c, ms] for st in info["trials"].values() for c, ms in st]}
        return dict(best)

    def configure(self, stereo, params, tune_missing: bool = True) -> dict | None:
        """Applies the tuned configuration to a CudaStereo handle (tuning first if `tune_missing`)."""
        kind = FrameKind.of(stereo.width, stereo.height, params)
        cfg = self.tune(kind, params=params) if tune_missing else self.lookup(kind)
        if cfg:
            apply(stereo, cfg)
        return cfg


_shared: Autotuner | None = None
_device: str | None = None


def tuned_config(width: int, height: int, params, batch: bool = False) -> dict | None:
    """The tuned configuration of this kind of frame on this GPU from the tables, or None (no tuning)."""
    global _shared, _device
    if _shared is None:
        _shared = Autotuner()
        _device = Autotuner.device_name()
    return _shared.lookup(FrameKind.of(width, height, params), _device, batch=batch)


def apply(stereo, cfg: dict) -> None:
    stereo.set_kernel_config(cfg["regs_per_lane"], cfg["lanes_per_line"], bool(cfg["materialize_costs"]),
                             cfg["path_warps_per_block"], cfg["wta_threads"], cfg["prefetch_steps"],
                             bool(cfg.get("fused_pairs", 0)), cfg.get("horz_warps_per_block", 4))


def device_timer(kind: FrameKind, frames: int, warmup: int, params=None):
    """time_fn for search(): one handle of this kind on a synthetic speckle pair; the device time of a frame
    (sum of its stage events, on the stream it runs on), median over `frames` frames."""
    import torch

    from .stereo import CudaStereo, SgmParams, StereoError, StereoParams
    from .synth import plane_sphere_pair
    dev = torch.device("cuda")
    pr = plane_sphere_pair(seed=7, width=kind.width, height=kind.height, f=1.4 * kind.width,
                           num_disparities=kind.num_disparities, device=dev)
    if params is None:
        params = StereoParams(sgm=SgmParams(min_disparity=pr.min_disparity, num_disparities=kind.num_disparities,
                                            eight_paths=kind.eight_paths), wide_costs=kind.wide)
    l = torch.from_numpy(pr.left).to(dev)
    r = torch.from_numpy(pr.right).to(dev)
    out = {"disparity_u16": torch.empty((kind.height, kind.width), dtype=torch.int16, device=dev)}
    st = torch.cuda.Stream(dev)
    s = CudaStereo.create(params, kind.width, kind.height)

    def time_fn(cfg: dict) -> float:
        try:
            apply(s, cfg)
        except StereoError:
            return float("inf")
        for _ in range(warmup):
            s.compute_device(l, r, out, stream=st)
        st.synchronize()
        s.profile(True)
        s.profile_collect()
        for _ in range(frames):
            s.compute_device(l, r, out, stream=st)
        rows = s.profile_collect()
        s.profile(False)
        return float(np.median(rows.sum(axis=1))) if len(rows) else float("inf")

    return time_fn


def batch_timer(kind: FrameKind, warmup: int, params=None, pairs: int = 8, reps: int = 3):
    """time_fn for the batched path: a StereoBatch of `pairs` frames of this kind with the library's default
    schedule; device time of one graph replay per frame, best of `reps`."""
    import torch

    from .batch import PairDesc, StereoBatch
    from .stereo import SgmParams, StereoError, StereoParams
    from .synth import plane_sphere_pair
    dev = torch.device("cuda")
    pr = plane_sphere_pair(seed=7, width=kind.width, height=kind.height, f=1.4 * kind.width,
                           num_disparities=kind.num_disparities, device=dev)
    if params is None:
        params = StereoParams(sgm=SgmParams(min_disparity=pr.min_disparity, num_disparities=kind.num_disparities,
                                            eight_paths=kind.eight_paths), wide_costs=kind.wide)
    l = torch.from_numpy(pr.left).to(dev)
    r = torch.from_numpy(pr.right).to(dev)
    outs = [{"disparity_u16": torch.empty((kind.height, kind.width), dtype=torch.int16, device=dev)} for _ in range(pairs)]
    st = torch.cuda.Stream(dev)

    def time_fn(cfg: dict) -> float:
        try:
            b = StereoBatch([PairDesc(kind.width, kind.height, params, kernel=cfg)] * pairs, tuned=False)
        except StereoError:
            return float("inf")
        try:
            for i, o in enumerate(outs):
                b.bind(i, l, r, o)
            for _ in range(max(warmup, 1)):
                b.run(stream=st)
            best = float("inf")
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st)
                b.run(stream=st)
                e1.record(st)
                e1.synchronize()
                best = min(best, e0.elapsed_time(e1) / pairs)
            return best
        finally:
            b.close()

    return time_fn


def batch_schedules(n_pairs: int) -> list[tuple[int, int]]:
    """(micro_batch, branches) candidates of a batch: all pairs per launch, and micro-batches on branches."""
    c = [(n_pairs, 1)]
    for mb in (1, 2, 4):
        for br in (2, 4, 8):
            if mb * br <= max(n_pairs, 2) * 2:
                c.append((mb, br))
    return c


def tune_batch_schedule(make_batch, run_fn, n_pairs: int, reps: int = 3) -> tuple[tuple[int, int], dict]:
    """Times each (micro_batch, branches) schedule. make_batch(mb, br) -> a bound StereoBatch;
    run_fn(batch) -> ms of one run. Returns the fastest schedule and all timings."""
    times = {}
    for mb, br in batch_schedules(n_pairs):
        b = make_batch(mb, br)
        try:
            run_fn(b)  # capture + warm-up
            times[(mb, br)] = min(run_fn(b) for _ in range(reps))
        finally:
            b.close()
    best = min(times, key=times.get)
    return best, times


def _parse_kind(s: str) -> FrameKind:
    size, rest = s.split(":")
    w, h = (int(v) for v in size.split("x"))
    parts = rest.split(",")
    d = int(parts[0])
    eight = "p8" in parts
    wide = "u16" in parts
    return FrameKind(w, h, d, eight, wide)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="Tune SGM kernel configurations on this GPU")
    ap.add_argument("kinds", nargs="+", help="WxH:D[,p8][,u16] frame kinds, e.g. 1280x1024:128 1280x1024:256,p8,u16")
    ap.add_argument("--write", action="store_true", help="write the packaged table (tuning/b200.json)")
    ap.add_argument("--frames", type=int, default=8)
    ap.add_argument("--batch", action="store_true", help="also tune for the batched path")
    args = ap.parse_args(argv)
    t = Autotuner(table_path=PACKAGE_TABLE if args.write else None, read_package_table=True)
    for ks in args.kinds:
        kind = _parse_kind(ks)
        for batch in ((False, True) if args.batch else (False,)):
            t0 = time.perf_counter()
            cfg = t.tune(kind, frames=args.frames, force=True, batch=batch)
            e = t.table[t._key(kind, t.device_name(), batch)]
            print(json.dumps({"kind": ks, "batch": batch, "config": cfg, "ms_per_frame": e["ms_per_frame"],
                              "tuning_s": time.perf_counter() - t0}), flush=True)
    if args.write:
        print("wrote", t.save(PACKAGE_TABLE))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
