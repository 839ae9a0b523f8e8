"""Offline re-depth (double-buffered batches of raw frames; 8 paths, 16-bit path values) against the
per-frame path, frame by frame, bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_offline_batches_equal_per_frame_runs(cuda):
    from open_source_einstar_b200 import CudaStereo, RectifiedGeometry, RemapTable, SgmParams, StereoParams, synth
    from open_source_einstar_b200.offline import OfflineRedepth
    w, h, d, n = 320, 256, 96, 8
    rec = synth.recording(n_frames=n, seed=3, width=w, height=h, f=275.0, num_disparities=d, device="cuda")
    frames = [synth.recording_frame(rec, i, device="cuda") for i in range(n)]
    lefts = np.stack([f[0] for f in frames])
    rights = np.stack([f[1] for f in frames])
    sp = StereoParams(sgm=SgmParams(min_disparity=rec.min_disparity, num_disparities=d, eight_paths=True),
                      wide_costs=True)
    geom = RectifiedGeometry(rec.rect.f, 0, 0, rec.rect.baseline, rec.rect.cx_offset)
    u16 = np.zeros((n, h, w), np.uint16)
    depth = np.zeros((n, h, w), np.float32)
    with OfflineRedepth(w, h, sp, rec.maps, (w, h), geom, batch_size=3) as off:  # 3 batches, the last partial
        st = off.run(lefts, rights, u16, depth)
        assert st.frames == n and st.batches == 3 and st.device_ms > 0
        st = off.run(lefts[::-1].copy(), rights[::-1].copy(), u16[::-1], depth[::-1])  # reused buffers
    (lx, ly), (rx, ry) = rec.maps
    with CudaStereo.create(sp, w, h) as s:
        s.set_rectification(RemapTable(lx, ly), RemapTable(rx, ry), w, h)
        s.set_point_params(geom, 150.0, 700.0)
        for i in range(n):
            r = s.compute_raw(lefts[i], rights[i])
            assert (r.disparity_u16 != 0xFFFF).mean() > 0.2, "too few valid pixels for a meaningful check"
            assert np.array_equal(r.disparity_u16, u16[i]), f"frame {i}"
            assert np.array_equal(r.depth.view(np.uint32), depth[i].view(np.uint32)), f"frame {i}"
