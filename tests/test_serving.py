"""Request server (ds_server_*): continuous batching of frames of mixed sizes and disparity ranges.

Each frame's result must be the same alone (CudaStereo.compute_raw, one frame on an idle GPU) and in the
mix (many frames admitted while others run, sharing slot volumes). Integer stages make this bit-exact;
the stated tolerances (1/64 px for u16 disparity, 1e-4 relative for depth) are asserted as well.
"""
import numpy as np
import pytest

from conftest import mismatch_report, same_bits

pytestmark = pytest.mark.gpu

DEPTH_RTOL = 1e-4
U16_TOL = 1

# (width, height, num_disparities) per calibration; two synthetic rigs per size
SIZES = [(320, 256, 64), (240, 192, 48), (160, 128, 32)]


def _rigs():
    from open_source_einstar_b200 import synth
    rigs = []
    for i, (w, h, d) in enumerate(SIZES):
        for k in range(2):
            pr = synth.raw_objects_pair(seed=200 + 2 * i + k, width=w, height=h, f=w * (0.8 + 0.1 * k),
                                        num_disparities=d, n_objects=6, device="cuda")
            rigs.append((w, h, d, pr))
    return rigs


def _frames(rigs, n, seed, pinned=True):
    """n requests drawn from the rigs (sizes mixed), each with its own output buffers (page-locked, so
    that frames overlap on the GPU; pageable for the rest)."""
    from open_source_einstar_b200 import SgmParams, StereoParams
    from open_source_einstar_b200.serving import pinned_copy, pinned_empty
    alloc = pinned_empty if pinned else np.empty
    rng = np.random.default_rng(seed)
    inputs = {}
    frames = []
    for i in range(n):
        c = int(rng.integers(len(rigs)))
        w, h, d, pr = rigs[c]
        if c not in inputs:
            inputs[c] = (pinned_copy(pr.left), pinned_copy(pr.right)) if pinned else (pr.left, pr.right)
        sp = StereoParams(sgm=SgmParams(min_disparity=pr.min_disparity, num_disparities=d))
        outs = {"disparity": alloc((h, w), np.float32), "disparity_u16": alloc((h, w), np.uint16),
                "depth": alloc((h, w), np.float32)}
        frames.append({"left": inputs[c][0], "right": inputs[c][1], "width": w, "height": h, "params": sp,
                       "outputs": outs, "calib": c})
    return frames


def _alone(rigs):
    from open_source_einstar_b200 import CudaStereo, RectifiedGeometry, RemapTable, SgmParams, StereoParams
    want = []
    for w, h, d, pr in rigs:
        (lx, ly), (rx, ry) = pr.maps
        sp = StereoParams(sgm=SgmParams(min_disparity=pr.min_disparity, num_disparities=d))
        with CudaStereo.create(sp, w, h) as s:
            s.set_rectification(RemapTable(lx, ly), RemapTable(rx, ry), w, h)
            s.set_point_params(RectifiedGeometry(pr.f, 0, 0, pr.baseline, pr.cx_offset), 150.0, 700.0)
            want.append(s.compute_raw(pr.left, pr.right))
    return want


def _server(rigs, **kw):
    from open_source_einstar_b200 import RectifiedGeometry, RemapTable
    from open_source_einstar_b200.serving import StereoServer
    srv = StereoServer(**kw)
    for c, (w, h, d, pr) in enumerate(rigs):
        (lx, ly), (rx, ry) = pr.maps
        srv.add_calibration(c, RemapTable(lx, ly), RemapTable(rx, ry), w, h,
                            RectifiedGeometry(pr.f, 0, 0, pr.baseline, pr.cx_offset), 150.0, 700.0)
    return srv


def _check(frames, want, completions):
    for i, f in enumerate(frames):
        assert completions[i].ok, f"frame {i} failed with status {completions[i].status}"
        w = want[f["calib"]]
        o = f["outputs"]
        assert same_bits(o["disparity"], w.disparity), f"frame {i}: {mismatch_report(o['disparity'], w.disparity)}"
        du = np.abs(o["disparity_u16"].astype(np.int64) - w.disparity_u16.astype(np.int64))
        assert du.max() <= U16_TOL and np.array_equal(o["disparity_u16"], w.disparity_u16)
        assert np.allclose(o["depth"], w.depth, rtol=DEPTH_RTOL, atol=0) and same_bits(o["depth"], w.depth)


def test_server_results_same_alone_and_in_the_mix(cuda):
    from open_source_einstar_b200.serving import poisson_arrivals, replay
    rigs = _rigs()
    want = _alone(rigs)
    with _server(rigs, max_slots=4) as srv:
        # a burst: every frame queued at once, admitted as slots free up, overlapping on the GPU
        frames = _frames(rigs, 36, seed=1)
        tickets = [srv.submit(f["left"], f["right"], f["width"], f["height"], f["params"], f["outputs"], f["calib"],
                              tag=i) for i, f in enumerate(frames)]
        done = srv.wait_all(tickets)
        _check(frames, want, [done[t] for t in tickets])
        st = srv.stats()
        assert st["completed"] == 36 and st["failed"] == 0 and st["peak_running"] > 1
        assert st["slots"] <= 4
        # Poisson arrivals at a high rate: frames arrive while others are on the GPU
        frames = _frames(rigs, 48, seed=2)
        comps, _ = replay(srv, frames, poisson_arrivals(2000.0, 48 / 2000.0 * 1.2, seed=3)[:48])
        by_tag = {c.tag: c for c in comps}
        _check(frames[:len(by_tag)], want, [by_tag[i] for i in range(len(by_tag))])


def test_server_admits_by_volume_budget(cuda):
    from open_source_einstar_b200 import SgmParams, StereoParams
    rigs = _rigs()[:2]  # 320x256, D=64
    want = _alone(rigs)
    w, h, d, pr = rigs[0]
    one = w * h * 64 * 4 + w * h * 64  # u8 path values of 4 directions + the u8 cost volume
    budget = int(2.5 * one)
    with _server(rigs, max_slots=8, volume_budget_bytes=budget) as srv:
        frames = _frames(rigs, 20, seed=4, pinned=False)  # pageable host buffers work too
        tickets = [srv.submit(f["left"], f["right"], f["width"], f["height"], f["params"], f["outputs"], f["calib"])
                   for f in frames]
        done = srv.wait_all(tickets)
        _check(frames, want, [done[t] for t in tickets])
        st = srv.stats()
        assert st["volume_bytes"] <= budget and st["peak_running_volume_bytes"] <= budget
        assert st["peak_running"] <= 2
        # a frame whose volume alone exceeds the budget completes with invalid_argument
        big = StereoParams(sgm=SgmParams(min_disparity=pr.min_disparity, num_disparities=256))
        out = {"disparity": np.empty((h, w), np.float32)}
        t = srv.submit(pr.left, pr.right, w, h, big, out, calib=0)
        c = srv.wait_all([t])[t]
        assert c.status == 5


def test_server_rejects_bad_requests(cuda):
    from open_source_einstar_b200 import Errc, SgmParams, StereoError, StereoParams
    rigs = _rigs()[:1]
    w, h, d, pr = rigs[0]
    sp = StereoParams(sgm=SgmParams(min_disparity=pr.min_disparity, num_disparities=d))
    with _server(rigs) as srv:
        out = {"disparity": np.empty((h, w), np.float32)}
        with pytest.raises(StereoError) as e:
            srv.submit(pr.left, pr.right, w, h, sp, out, calib=7)  # unknown calibration
        assert e.value.code == Errc.invalid_argument
        with pytest.raises(StereoError):
            srv.submit(pr.left, pr.right, w + 8, h, sp, {"disparity": np.empty((h, w + 8), np.float32)},
                       calib=0)  # remap size matches neither the frame size nor twice it
        with pytest.raises(StereoError):
            srv.submit(pr.left, pr.right, w, h, sp, {"depth": np.empty((h, w), np.float32)}, calib=-1)  # no geometry
        bad = StereoParams(sgm=SgmParams(num_disparities=600))
        with pytest.raises(StereoError) as e:
            srv.submit(pr.left, pr.right, w, h, bad, out, calib=0)
        assert e.value.code == Errc.invalid_argument
        assert srv.stats()["submitted"] == 0


def test_server_config4_sizes_against_the_reference(cuda, ref, port):
    """Frames of configuration 4's three sizes (1280x1024 D=128, 960x768 D=96, 640x512 D=96; raw pairs, GPU
    remap) queued together on the server: each result equals the reference pipeline directly (the restated
    remap, the reference's sgm_disparity + median3, the restated depth), not only a per-frame CUDA run."""
    from open_source_einstar_b200 import SgmParams, StereoParams, synth
    from oracle.oracle import OracleSgm
    specs = [(1280, 1024, 128), (960, 768, 96), (640, 512, 96)]
    rigs = []
    for i, (w, h, d) in enumerate(specs):
        pr = synth.raw_objects_pair(seed=300 + i, width=w, height=h, f=1100.0 * w / 1280, num_disparities=d,
                                    device="cuda")
        rigs.append((w, h, d, pr))
    with _server(rigs, max_slots=3) as srv:
        frames = _frames(rigs, 6, seed=7)
        for c in range(len(rigs)):  # every size at least once
            frames[c] = _frames([rigs[c]], 1, seed=c)[0]
            frames[c]["calib"] = c
        tickets = [srv.submit(f["left"], f["right"], f["width"], f["height"], f["params"], f["outputs"], f["calib"],
                              tag=i) for i, f in enumerate(frames)]
        done = srv.wait_all(tickets)
    want = {}
    for c, (w, h, d, pr) in enumerate(rigs):
        (lx, ly), (rx, ry) = pr.maps
        p = OracleSgm(min_disparity=pr.min_disparity, num_disparities=d)
        rl, rr = port.remap(pr.left, lx, ly), port.remap(pr.right, rx, ry)
        disp = ref.median3(ref.sgm_disparity(rl, rr, p))
        want[c] = (disp, port.encode_u16(disp, p.min_disparity),
                   port.depth(disp, pr.f, pr.baseline, pr.cx_offset, 150.0, 700.0))
    for i, (f, t) in enumerate(zip(frames, tickets)):
        assert done[t].ok, f"frame {i}: status {done[t].status}"
        disp, u16, z = want[f["calib"]]
        o = f["outputs"]
        assert same_bits(o["disparity"], disp), f"frame {i} ({f['width']}x{f['height']}): {mismatch_report(o['disparity'], disp)}"
        assert np.array_equal(o["disparity_u16"], u16)
        nz = z > 0
        assert np.all(np.abs(o["depth"][nz] - z[nz]) <= DEPTH_RTOL * z[nz]) and same_bits(o["depth"], z)
