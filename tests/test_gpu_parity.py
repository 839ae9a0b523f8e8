"""Parity of the CUDA path (through the C ABI) with the oracle: bit-exact integer and float stages.

The reference's own GPU-vs-CPU test allows 0.25 px (tests/depth/test_metal_stereo.cpp:120); this path
is held to bit-identical disparities. Depth is computed in double like the reference and is compared
bit-for-bit too (the stated tolerance, 1e-4 relative, is asserted as well).
"""
import hashlib

import numpy as np
import pytest

from conftest import mismatch_report, same_bits
from oracle.oracle import OracleSgm

pytestmark = pytest.mark.gpu

DEPTH_RTOL = 1e-4        # stated tolerance for depth (relative)
U16_TOL = 1              # 1/64 px: the u16 encoding's step


def _stereo(params: OracleSgm, w, h, subpixel=True, median=False, wide=False):
    from open_source_einstar_b200 import CudaStereo, SgmParams, StereoParams
    sp = StereoParams(sgm=SgmParams(**params.__dict__), subpixel=subpixel, median=median, wide_costs=wide)
    return CudaStereo.create(sp, w, h)


def test_golden_cases_bit_exact(cuda, golden):
    for name, c in golden.items():
        p = OracleSgm(**c["params"])
        h, w = c["shape"]
        with _stereo(p, w, h, c["subpixel"], median=False) as s:
            r = s.compute(c["left"], c["right"])
            if "disparity" in c:
                assert same_bits(r.disparity, c["disparity"]), f"{name}: {mismatch_report(r.disparity, c['disparity'])}"
            else:
                assert hashlib.sha256(r.disparity.tobytes()).hexdigest() == c["disparity_sha256"], name
            assert np.array_equal(r.confidence, (r.disparity > -1e8).astype(np.float32))
            if "census_left" in c:
                cl, _, _ = s.debug_read(census=True, sums=False)
                assert same_bits(cl, c["census_left"]), name
        with _stereo(p, w, h, c["subpixel"], median=True) as s:
            r = s.compute(c["left"], c["right"])
            if "median" in c:
                assert same_bits(r.disparity, c["median"]), f"{name} (median): {mismatch_report(r.disparity, c['median'])}"
            else:
                assert hashlib.sha256(r.disparity.tobytes()).hexdigest() == c["median_sha256"], name


def test_path_sums_match_oracle(cuda, golden, port):
    """Stage check: the summed path costs (the reference's u16 `sum` volume) are identical."""
    for name in ("plane_sphere_160x128", "eight_paths", "census_9x7_wide", "tiny_37x29_d5", "d_not_multiple_of_32_d40"):
        c = golden[name]
        p = OracleSgm(**c["params"])
        h, w = c["shape"]
        with _stereo(p, w, h) as s:
            s.compute(c["left"], c["right"])
            cl, cr, sums = s.debug_read()
        cost = port.cost_volume(port.census(c["left"], p.census_radius_x, p.census_radius_y),
                                port.census(c["right"], p.census_radius_x, p.census_radius_y), p)
        want = port.aggregate(cost, c["left"], p)
        assert same_bits(sums, want), f"{name}: {mismatch_report(sums, want)}"


@pytest.mark.parametrize("seed", [0, 1])
def test_config1_plane_sphere_full_outputs(cuda, port, seed):
    """640x512, D=64, default SGM: u16 disparity and f32 depth against the oracle pipeline."""
    from open_source_einstar_b200 import RectifiedGeometry, synth
    pair = synth.plane_sphere_pair(seed=seed)
    p = OracleSgm(min_disparity=pair.min_disparity, num_disparities=pair.num_disparities)
    want = port.pipeline(pair.left, pair.right, p, median=True, geometry=(pair.f, pair.baseline, 0.0))
    with _stereo(p, 640, 512, median=True) as s:
        s.set_point_params(RectifiedGeometry(pair.f, 319.5, 255.5, pair.baseline, 0.0), 150.0, 700.0)
        r = s.compute(pair.left, pair.right)
        t = s.last_timings()
    assert same_bits(r.disparity, want["disparity"]), mismatch_report(r.disparity, want["disparity"])
    assert np.array_equal(r.disparity_u16, want["disparity_u16"])
    assert np.abs(r.disparity_u16.astype(int) - want["disparity_u16"].astype(int)).max() <= U16_TOL
    zw, zg = want["depth"], r.depth
    assert np.array_equal(zg > 0, zw > 0)
    nz = zw > 0
    assert np.all(np.abs(zg[nz] - zw[nz]) <= DEPTH_RTOL * zw[nz])
    assert same_bits(zg, zw)
    assert (r.disparity > -1e8).mean() > 0.6
    assert t.gpu_ms > 0 and t.total_ms >= t.gpu_ms


def test_config2_raw_1280x1024_d128(cuda, ref, port):
    """Raw distorted pair -> GPU remap (bit-exact rectified bytes) -> SGM D=128 -> L-R -> median -> depth."""
    from open_source_einstar_b200 import CudaStereo, RectifiedGeometry, RemapTable, SgmParams, StereoParams, synth
    pair = synth.raw_objects_pair(seed=0, device="cuda")
    (lx, ly), (rx, ry) = pair.maps
    p = OracleSgm(min_disparity=pair.min_disparity, num_disparities=128)
    with CudaStereo.create(StereoParams(sgm=SgmParams(**p.__dict__)), 1280, 1024) as s:
        s.set_rectification(RemapTable(lx, ly), RemapTable(rx, ry), 1280, 1024)
        s.set_point_params(RectifiedGeometry(pair.f, 0, 0, pair.baseline, 0.0), 150.0, 700.0)
        r = s.compute_raw(pair.left, pair.right, rectified=True)
    rl, rr = port.remap(pair.left, lx, ly), port.remap(pair.right, rx, ry)
    assert np.array_equal(r.rect_left, rl) and np.array_equal(r.rect_right, rr)  # test_metal_stereo.cpp:103
    d = ref.median3(ref.sgm_disparity(rl, rr, p))
    assert same_bits(r.disparity, d), mismatch_report(r.disparity, d)
    z = port.depth(d, pair.f, pair.baseline, 0.0, 150.0, 700.0)
    assert same_bits(r.depth, z)


def test_half_resolution_rectification(cuda, port):
    """Remap tables at twice the stereo size: remap + 2x2 box average (calib::remap + depth::downsample2)."""
    from open_source_einstar_b200 import CudaStereo, RemapTable, SgmParams, StereoParams, synth
    pair = synth.raw_objects_pair(seed=3, width=320, height=256, f=275.0, num_disparities=32, n_objects=8, device="cuda")
    (lx, ly), (rx, ry) = pair.maps
    p = OracleSgm(min_disparity=pair.min_disparity // 2, num_disparities=32)
    with CudaStereo.create(StereoParams(sgm=SgmParams(**p.__dict__)), 160, 128) as s:
        s.set_rectification(RemapTable(lx, ly), RemapTable(rx, ry), 320, 256)
        r = s.compute_raw(pair.left, pair.right, rectified=True)

    def down(img):
        a = img.astype(np.int32)
        return ((a[0::2, 0::2] + a[0::2, 1::2] + a[1::2, 0::2] + a[1::2, 1::2] + 2) // 4).astype(np.uint8)

    hl, hr = down(port.remap(pair.left, lx, ly)), down(port.remap(pair.right, rx, ry))
    assert np.array_equal(r.rect_left, hl) and np.array_equal(r.rect_right, hr)
    assert same_bits(r.disparity, port.median3(port.sgm_disparity(hl, hr, p)))


def test_wide_eight_path_d256(cuda, port):
    """The offline configuration's arithmetic at a small size: 8 paths, D=256, 16-bit path values."""
    from open_source_einstar_b200 import synth
    pair = synth.plane_sphere_pair(seed=5, width=320, height=200, f=450.0, num_disparities=256)
    p = OracleSgm(min_disparity=max(pair.min_disparity - 60, 0), num_disparities=256, eight_paths=True)
    with _stereo(p, 320, 200, median=True, wide=True) as s:
        r = s.compute(pair.left, pair.right)
    want = port.median3(port.sgm_disparity(pair.left, pair.right, p))
    assert same_bits(r.disparity, want), mismatch_report(r.disparity, want)


def test_repeated_frames_bit_identical(cuda, golden):
    """tests/depth/test_metal_stereo.cpp:157: repeated frames give identical bytes."""
    c = golden["plane_sphere_160x128"]
    p = OracleSgm(**c["params"])
    with _stereo(p, 160, 128, median=True) as s:
        outs = [s.compute(c["left"], c["right"]) for _ in range(3)]
    for o in outs[1:]:
        assert same_bits(o.disparity, outs[0].disparity) and np.array_equal(o.disparity_u16, outs[0].disparity_u16)


def test_device_entry_matches_host_entry(cuda, golden):
    import torch
    c = golden["plane_sphere_160x128"]
    p = OracleSgm(**c["params"])
    with _stereo(p, 160, 128, median=True) as s:
        host = s.compute(c["left"], c["right"])
        l = torch.from_numpy(c["left"]).cuda()
        r = torch.from_numpy(c["right"]).cuda()
        out = {"disparity": torch.empty((128, 160), dtype=torch.float32, device="cuda"),
               "disparity_u16": torch.empty((128, 160), dtype=torch.int16, device="cuda")}
        st = torch.cuda.current_stream()
        s.compute_device(l, r, out, stream=st)
        st.synchronize()
    assert same_bits(out["disparity"].cpu().numpy(), host.disparity)
    assert np.array_equal(out["disparity_u16"].cpu().numpy().view(np.uint16), host.disparity_u16)


def test_stage_profile(cuda, golden):
    """Per-frame stage times (the reference's per-stage GPU profile): one row per frame, the cost stage
    empty when the path kernels recompute costs, and profiling leaves the results unchanged."""
    from open_source_einstar_b200.stereo import STAGE_NAMES
    c = golden["plane_sphere_160x128"]
    p = OracleSgm(**c["params"])
    with _stereo(p, 160, 128) as s:
        s.set_kernel_config(1, 16, materialize_costs=True)
        s.profile(True)
        outs = [s.compute(c["left"], c["right"]) for _ in range(3)]
        rows = s.profile_collect()
        s.set_kernel_config(1, 16, materialize_costs=False)
        outs.append(s.compute(c["left"], c["right"]))
        rows2 = s.profile_collect()
    assert rows.shape == (3, len(STAGE_NAMES)) and rows2.shape == (1, len(STAGE_NAMES))
    costs, paths = STAGE_NAMES.index("costs"), STAGE_NAMES.index("paths")
    assert (rows >= 0).all() and (rows[:, costs] > 0).all() and (rows[:, paths] > 0).all()
    assert rows2[0, costs] < 0.01 and rows2[0, paths] > 0
    for o in outs:
        assert same_bits(o.disparity, c["disparity"])


def test_strided_host_images(cuda, golden):
    c = golden["plane_sphere_160x128"]
    p = OracleSgm(**c["params"])
    big_l = np.zeros((128, 200), np.uint8)
    big_r = np.zeros((128, 200), np.uint8)
    big_l[:, 10:170] = c["left"]
    big_r[:, 10:170] = c["right"]
    with _stereo(p, 160, 128) as s:
        r = s.compute(big_l[:, 10:170], big_r[:, 10:170])
    assert same_bits(r.disparity, c["disparity"])


def test_errors_follow_the_reference(cuda, golden):
    from open_source_einstar_b200 import Errc, StereoError
    c = golden["plane_sphere_160x128"]
    p = OracleSgm(**c["params"])
    with _stereo(p, 160, 128) as s:
        with pytest.raises(StereoError) as e:
            s.compute(c["left"][:100], c["right"][:100])  # metal_stereo.cpp:235-236
        assert e.value.code == Errc.invalid_argument
        with pytest.raises(StereoError) as e:
            s.compute_raw(c["left"], c["right"])  # metal_stereo.cpp:343
        assert e.value.code == Errc.invalid_argument and "set_rectification" in e.value.message
        from open_source_einstar_b200 import RemapTable
        m = np.zeros((100, 100), np.float32)
        with pytest.raises(StereoError) as e:
            s.set_rectification(RemapTable(m, m), RemapTable(m, m), 100, 100)  # metal_stereo.cpp:205-206
        assert e.value.code == Errc.invalid_argument
        # the handle stays usable after rejected calls
        r = s.compute(c["left"], c["right"])
        assert same_bits(r.disparity, c["disparity"])


SUPPORTED = [(r, 8) for r in (4, 6, 8)] + [(r, 16) for r in (1, 2, 3, 4)] + [(r, 32) for r in (1, 2, 3, 4, 6, 8)]
SWEEP = [(6, 4), (8, 4), (6, 8), (8, 8)]  # (regs per lane, lanes per line) of the sweep kernels


def _sweep_fit(p: OracleSgm, w, h):
    from open_source_einstar_b200 import SgmParams, StereoParams
    from open_source_einstar_b200.autotune import FrameKind
    return FrameKind.of(w, h, StereoParams(sgm=SgmParams(**p.__dict__))).sweep_fit()


@pytest.mark.parametrize("mode", ["per_direction", "materialized", "fused_pairs"])
def test_every_kernel_config_is_bit_exact(cuda, golden, port, mode):
    """All (lanes per line, regs per lane) configurations and all SGM kernel modes give identical bytes;
    fused_pairs runs the sweep kernels in each of their shapes."""
    for name in ("plane_sphere_160x128", "d_not_multiple_of_32_d40", "eight_paths", "census_9x7_wide", "tiny_37x29_d5",
                 "census_7x7_u64", "negative_min_disparity", "no_subpixel_uniq08_lr2", "no_slant_fixed_p2",
                 "unmatched_noise"):
        c = golden[name]
        p = OracleSgm(**c["params"])
        h, w = c["shape"]
        if mode == "fused_pairs" and not _sweep_fit(p, w, h):
            continue
        want = c["median"]
        for r, seg in (SWEEP if mode == "fused_pairs" else SUPPORTED):
            if 2 * r * seg < p.num_disparities:
                continue
            for pf in ((4,) if mode == "fused_pairs" else (4, 8)):
                with _stereo(p, w, h, c["subpixel"], median=True) as s:
                    s.set_kernel_config(r, seg, mode == "materialized", path_warps_per_block=2 if r > 4 else 4,
                                        wta_threads=128, prefetch_steps=pf, fused_pairs=mode == "fused_pairs",
                                        horz_warps_per_block=2)
                    got = s.compute(c["left"], c["right"]).disparity
                assert same_bits(got, want), f"{name} R={r} SEG={seg} {mode} PF={pf}: {mismatch_report(got, want)}"


@pytest.mark.parametrize("w,h,nd,mind", [(75, 41, 24, 3), (33, 7, 40, 0), (129, 2, 16, 5), (1, 9, 4, 0), (9, 1, 4, 0)])
def test_odd_and_degenerate_sizes(cuda, port, w, h, nd, mind):
    """Odd sizes split the meet-in-the-middle sweeps unevenly; 1-pixel rows/columns have one-step lines."""
    rng = np.random.default_rng(w * 1000 + h)
    base = (rng.random((h, w + 40)) * 255).astype(np.uint8)
    left = base[:, 20:20 + w].copy()
    right = base[:, 14:14 + w].copy()
    p = OracleSgm(min_disparity=mind, num_disparities=nd)
    want = port.median3(port.sgm_disparity(left, right, p))
    from open_source_einstar_b200.autotune import sweep_shapes
    for fused in (False, True):
        with _stereo(p, w, h, median=True) as s:
            cfg = s.kernel_config()
            r, seg = sweep_shapes(nd)[0] if fused else (cfg["regs_per_lane"], cfg["lanes_per_line"])
            s.set_kernel_config(r, seg, False, 1, 64, 4, fused, 1)
            got = s.compute(left, right).disparity
        assert same_bits(got, want), f"{w}x{h} fused={fused}: {mismatch_report(got, want)}"


def test_batch_matches_per_pair_runs(cuda, port):
    """Uneven sizes and disparity ranges, rectified and raw pairs (two calibrations), kernel variants:
    one batched graph launch equals per-pair runs bit for bit, also after replay and re-binding."""
    import torch
    from open_source_einstar_b200 import (CudaStereo, PairDesc, RectifiedGeometry, RemapTable, SgmParams, StereoBatch,
                                          StereoParams, synth)
    sweep = {"fused_pairs": 1, "materialize_costs": 0}
    specs = [(320, 256, 64, None), (160, 128, 96, None), (240, 192, 128, None), (200, 136, 192, None),
             (160, 128, 40, {"regs_per_lane": 3, "lanes_per_line": 16, "materialize_costs": 0}),
             (128, 96, 64, {"regs_per_lane": 1, "lanes_per_line": 32, "materialize_costs": 1, "prefetch_steps": 8}),
             (240, 192, 128, {"regs_per_lane": 8, "lanes_per_line": 8, **sweep}),
             (160, 128, 40, {"regs_per_lane": 6, "lanes_per_line": 4, **sweep}),
             (200, 136, 96, {"regs_per_lane": 6, "lanes_per_line": 8, **sweep})]
    rect_pairs = [synth.plane_sphere_pair(seed=40 + i, width=w, height=h, f=w * 1.4, num_disparities=d)
                  for i, (w, h, d, _) in enumerate(specs)]
    raw_specs = [(256, 192, 0, None), (256, 192, 0, {"regs_per_lane": 8, "lanes_per_line": 4, **sweep}), (192, 160, 1, None)]
    raw_pairs = [synth.raw_objects_pair(seed=60 + i, width=w, height=h, f=w * 0.86, num_disparities=64, n_objects=6,
                                        device="cuda") for i, (w, h, _, _) in enumerate(raw_specs)]
    descs, inputs, want = [], [], []
    for (w, h, d, k), pr in zip(specs, rect_pairs):
        sp = StereoParams(sgm=SgmParams(min_disparity=pr.min_disparity, num_disparities=d))
        descs.append(PairDesc(w, h, sp, geometry=RectifiedGeometry(pr.f, 0, 0, pr.baseline), kernel=k))
        inputs.append((pr.left, pr.right))
    calibs = {}
    first_raw = len(descs)
    for (w, h, ci, k), pr in zip(raw_specs, raw_pairs):
        sp = StereoParams(sgm=SgmParams(min_disparity=pr.min_disparity, num_disparities=64))
        descs.append(PairDesc(w, h, sp, raw=True, calib=ci, kernel=k))
        inputs.append((pr.left, pr.right))
        calibs.setdefault(ci, (pr.maps, w, h))
    for d, (l, r), i in zip(descs, inputs, range(len(descs))):
        with CudaStereo.create(d.params, d.width, d.height) as s:
            if d.kernel:
                kk = {"path_warps_per_block": 4, "wta_threads": 256, "prefetch_steps": 4, **d.kernel}
                s.set_kernel_config(kk["regs_per_lane"], kk["lanes_per_line"], bool(kk.get("materialize_costs", 0)),
                                    kk["path_warps_per_block"], kk["wta_threads"], kk["prefetch_steps"],
                                    bool(kk.get("fused_pairs", 0)))
            if d.raw:
                (mlx, mly), (mrx, mry) = calibs[d.calib][0]
                s.set_rectification(RemapTable(mlx, mly), RemapTable(mrx, mry), d.width, d.height)
                res = s.compute_raw(l, r)
            else:
                if d.geometry is not None:
                    s.set_point_params(d.geometry, d.min_depth, d.max_depth)
                res = s.compute(l, r)
        want.append(res)
    volume_bytes = []
    for micro_batch, branches in ((len(descs), 1), (0, 0)):  # all pairs per launch; the default schedule
        b = StereoBatch(descs, n_calib=2, micro_batch=micro_batch, branches=branches)
        volume_bytes.append(b.device_bytes)
        for ci, ((mlx, mly), (mrx, mry)), w, h in [(ci, v[0], v[1], v[2]) for ci, v in calibs.items()]:
            b.set_rectification(ci, RemapTable(mlx, mly), RemapTable(mrx, mry), w, h)
        dev_in, dev_out = [], []
        for i, (l, r) in enumerate(inputs):
            dl, dr = torch.from_numpy(l).cuda(), torch.from_numpy(r).cuda()
            o = {"disparity": torch.empty(l.shape, dtype=torch.float32, device="cuda"),
                 "disparity_u16": torch.empty(l.shape, dtype=torch.int16, device="cuda")}
            if descs[i].geometry is not None:
                o["depth"] = torch.empty(l.shape, dtype=torch.float32, device="cuda")
            b.bind(i, dl, dr, o)
            dev_in.append((dl, dr))
            dev_out.append(o)
        st = torch.cuda.current_stream()
        for rep in range(2):
            for o in dev_out:
                o["disparity"].fill_(7.0)
            b.run(stream=st)
            st.synchronize()
            for i, (o, wres) in enumerate(zip(dev_out, want)):
                got = o["disparity"].cpu().numpy()
                assert same_bits(got, wres.disparity), f"pair {i} rep {rep}: {mismatch_report(got, wres.disparity)}"
                assert np.array_equal(o["disparity_u16"].cpu().numpy().view(np.uint16), wres.disparity_u16)
                if "depth" in o:
                    assert same_bits(o["depth"].cpu().numpy(), wres.depth)
        # re-bind: the first raw pair takes the second's inputs (same size and calibration; the second runs on
        # the sweep kernels); the captured graph is replayed
        b.bind(first_raw, dev_in[first_raw + 1][0], dev_in[first_raw + 1][1], dev_out[first_raw])
        b.run(stream=st)
        st.synchronize()
        assert same_bits(dev_out[first_raw]["disparity"].cpu().numpy(), want[first_raw + 1].disparity)
        # re-bind a rectified sweep pair to new buffers with its inputs and scribble over the old ones: the
        # sweep kernels' guide (the census kernel's copy of the left image) follows the binding
        nl, nr = dev_in[6][0].clone(), dev_in[6][1].clone()
        b.bind(6, nl, nr, dev_out[6])
        dev_in[6][0].fill_(77)
        dev_in[6][1].fill_(13)
        b.run(stream=st)
        st.synchronize()
        assert same_bits(dev_out[6]["disparity"].cpu().numpy(), want[6].disparity)
        if branches == 1:  # one persistent launch per stage and kernel variant for all pairs
            assert b.launches_per_run < 5 * len(descs) // 2
        b.close()
    # micro-batches that run one after another on a branch share their cost and path-value volumes
    assert volume_bytes[1] < volume_bytes[0]
