"""Autotuner (host logic on CPU; one small tuning run on the GPU)."""
import json

import numpy as np
import pytest

from open_source_einstar_b200.autotune import (SUPPORTED, SWEEP_SHAPES, Autotuner, FrameKind, batch_schedules, search,
                                               stage_candidates, sweep_shapes, tile_shapes)


@pytest.mark.parametrize("d", [4, 16, 24, 32, 40, 64, 96, 128, 192, 256, 384, 512])
def test_tile_shapes_cover_the_disparities_with_least_padding(d):
    shapes = tile_shapes(d)
    assert shapes
    for r, seg in shapes:
        assert r in SUPPORTED[seg] and seg * 2 * r >= d
        smaller = [x for x in SUPPORTED[seg] if x < r]
        assert all(seg * 2 * x < d for x in smaller)


def test_staged_search_finds_the_fastest_of_each_stage():
    kind = FrameKind(1280, 1024, 128, eight_paths=True)  # the per-pixel WTA: its block size is searched too
    # a synthetic cost model: SEG 16 R4 materialised, 8 warps, prefetch 8, 128-thread WTA is fastest
    def cost(c):
        ms = 1.0
        ms += 0.0 if (c["regs_per_lane"], c["lanes_per_line"]) == (4, 16) else 0.3
        ms += 0.0 if c["materialize_costs"] else 0.8
        ms += 0.5 if c.get("fused_pairs") else 0.0
        ms += {1: 0.05, 2: 0.04, 4: 0.03, 8: 0.0}[c["path_warps_per_block"]]
        ms += 0.0 if c["prefetch_steps"] == 8 else 0.02
        ms += 0.0 if c["wta_threads"] == 128 else 0.01
        return ms
    best, info = search(kind, cost)
    assert best == {"regs_per_lane": 4, "lanes_per_line": 16, "materialize_costs": 1, "path_warps_per_block": 8,
                    "wta_threads": 128, "prefetch_steps": 8, "fused_pairs": 0, "horz_warps_per_block": 4}
    assert info["ms"] == pytest.approx(1.0)
    n = sum(len(v) for v in info["trials"].values())
    assert n <= 30  # staged: two shapes go through the block search, not the full product (~100)
    # 4 paths, byte values, a 128-disparity slab: the row-sweep WTA, whose block shape is fixed
    row = FrameKind(1280, 1024, 128)
    best4 = {**best, "fused_pairs": 0}
    assert row.row_wta_fit(128) and stage_candidates(row, 3, best4) == [best4]
    slab192 = {**best4, "regs_per_lane": 3, "lanes_per_line": 32}
    assert not row.row_wta_fit(192) and len(stage_candidates(row, 3, slab192)) == 2


@pytest.mark.parametrize("d", [4, 24, 40, 48, 64, 96, 128])
def test_sweep_shapes_cover_the_disparities_with_least_padding(d):
    shapes = sweep_shapes(d)
    assert shapes
    for r, seg in shapes:
        assert r in SWEEP_SHAPES[seg] and seg * 2 * r >= d
        assert all(seg * 2 * x < d for x in SWEEP_SHAPES[seg] if x < r)


def test_sweep_candidates_only_where_the_kernels_fit():
    from open_source_einstar_b200 import SgmParams, StereoParams
    fits = FrameKind.of(1280, 1024, StereoParams(sgm=SgmParams(num_disparities=128)))
    assert fits.sweep_fit()
    sweeps = [c for c in stage_candidates(fits, 1) if c.get("fused_pairs")]
    assert [(c["regs_per_lane"], c["lanes_per_line"]) for c in sweeps] == [(8, 8)]
    assert not [c for c in stage_candidates(fits, 1, fused_ok=False) if c.get("fused_pairs")]
    for sp in (SgmParams(num_disparities=128, eight_paths=True),          # 8 paths
               SgmParams(num_disparities=192),                            # D > 128
               SgmParams(num_disparities=64, p2=120),                     # 2 (window + P2) > 255
               SgmParams(num_disparities=64, census_radius_x=3, census_radius_y=3)):  # 48 neighbours
        kind = FrameKind.of(640, 512, StereoParams(sgm=sp))
        assert not kind.sweep_fit() and not [c for c in stage_candidates(kind, 1) if c.get("fused_pairs")]


def test_rejected_configurations_are_skipped():
    kind = FrameKind(640, 512, 64, eight_paths=True)
    assert all(not c.get("fused_pairs") for c in stage_candidates(kind, 1))  # the sweep kernels need 4 paths
    best, _ = search(kind, lambda c: float("inf") if c["lanes_per_line"] != 32 else 1.0)
    assert best["lanes_per_line"] == 32


def test_table_roundtrip(tmp_path):
    path = str(tmp_path / "t.json")
    t = Autotuner(table_path=path, read_package_table=False)
    kind = FrameKind(320, 256, 64)
    cfg = {"regs_per_lane": 2, "lanes_per_line": 16, "materialize_costs": 1, "path_warps_per_block": 8,
           "wta_threads": 256, "prefetch_steps": 8, "fused_pairs": 0, "horz_warps_per_block": 4}
    t.table[kind.key("GPU X")] = {"config": cfg, "ms_per_frame": 0.1, "trials": []}
    t.save()
    t2 = Autotuner(table_path=path, read_package_table=False)
    assert t2.lookup(kind, "GPU X") == cfg and t2.lookup(kind, "GPU Y") is None
    assert json.load(open(path))["format"] == 1


def test_frame_kind_from_params():
    from open_source_einstar_b200 import SgmParams, StereoParams
    k = FrameKind.of(1280, 1024, StereoParams(sgm=SgmParams(num_disparities=256, eight_paths=True, p2=300)))
    assert k == FrameKind(1280, 1024, 256, True, True, 25, False)


def test_batch_schedules():
    s = batch_schedules(16)
    assert (16, 1) in s and (1, 4) in s and len(set(s)) == len(s)


@pytest.mark.gpu
def test_tuning_on_the_device(cuda, tmp_path):
    from open_source_einstar_b200 import CudaStereo, SgmParams, StereoParams, synth
    t = Autotuner(table_path=str(tmp_path / "t.json"), read_package_table=False)
    kind = FrameKind(320, 256, 48)
    cfg = t.tune(kind, frames=3, warmup=1)
    e = t.table[kind.key(t.device_name())]
    assert np.isfinite(e["ms_per_frame"]) and e["ms_per_frame"] > 0 and len(e["trials"]) >= 8
    assert t.tune(kind) == cfg  # cached
    pr = synth.plane_sphere_pair(seed=3, width=320, height=256, f=450.0, num_disparities=48)
    sp = StereoParams(sgm=SgmParams(min_disparity=pr.min_disparity, num_disparities=48))
    with CudaStereo.create(sp, 320, 256) as a, CudaStereo.create(sp, 320, 256) as b:
        t.configure(b, sp, tune_missing=False)
        assert b.kernel_config()["regs_per_lane"] == cfg["regs_per_lane"]
        ra, rb = a.compute(pr.left, pr.right), b.compute(pr.left, pr.right)
    assert np.array_equal(ra.disparity.view(np.uint32), rb.disparity.view(np.uint32))
