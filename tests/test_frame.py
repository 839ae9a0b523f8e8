"""ds_compute_frame, the scanner frontend's per-frame call (MetalStereo::compute_frame,
libs/pipeline/src/stereo_frontend.cpp:302-328): a raw pair in, the frame's points, normals and weights left on
the device, the marker candidates handed over early. Checked against the separate calls it combines
(compute_raw, disparity_to_points, compute_raw with blobs), and against the oracle's points."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_compute_frame_equals_the_separate_calls(cuda, port):
    import torch
    from open_source_einstar_b200 import (BlobParams, CudaStereo, PointImageParams, RectifiedGeometry, RemapTable, SgmParams,
                                          StereoParams, disparity_to_points, synth)
    pr = synth.raw_objects_pair(seed=8, width=640, height=512, f=560.0, num_disparities=64, n_objects=8, device="cuda")
    left, _ = synth.add_markers((pr.left * 0.6).astype(np.uint8), n_markers=12, seed=3)
    right, _ = synth.add_markers((pr.right * 0.6).astype(np.uint8), n_markers=12, seed=4)
    (lx, ly), (rx, ry) = pr.maps
    w, h = 320, 256
    # the frontend's configuration: half-resolution stereo with depth::compute_disparity's stages
    sp = StereoParams(sgm=SgmParams(min_disparity=pr.min_disparity // 4 - 2, num_disparities=40), pyramid_levels=1, median=False,
                      detail_enabled=True, filter_occlusion=True, filter_spikes=True, speckle_max_region_size=100)
    half = RectifiedGeometry(pr.f / 2, (w - 1) / 2.0, (h - 1) / 2.0, pr.baseline, 0.0)
    with CudaStereo.create(sp, w, h) as s:
        s.set_rectification(RemapTable(lx, ly), RemapTable(rx, ry), 640, 512)
        s.set_point_params(half, 150.0, 700.0, 4.0)
        s.set_blob_params(BlobParams())
        ref = s.compute_raw(left, right, blobs=True)
        pts = torch.zeros((h, w, 4), dtype=torch.float32, device=cuda)
        nrm = torch.zeros((h, w, 4), dtype=torch.float32, device=cuda)
        wts = torch.zeros((h, w), dtype=torch.float32, device=cuda)
        seen = []
        for _ in range(2):
            r = s.compute_frame(left, right, pts, nrm, wts, blobs=True, on_blobs=lambda a, b: seen.append((a, b)))
            assert np.array_equal(r.disparity.view(np.uint32), ref.disparity.view(np.uint32))
            assert np.array_equal(r.confidence.view(np.uint32), ref.confidence.view(np.uint32))
            for side in (0, 1):
                assert np.array_equal(r.blobs[side], ref.blobs[side])
                assert np.array_equal(seen[-1][side], ref.blobs[side])
        assert len(seen) == 2 and len(ref.blobs[0]) >= 12
        d = torch.from_numpy(ref.disparity).to(cuda)
        c = torch.from_numpy(ref.confidence).to(cuda)
        want = disparity_to_points(d, c, half, PointImageParams(150.0, 700.0, 4.0))
        torch.cuda.synchronize()
        for got, key in ((pts, "points"), (nrm, "normals"), (wts, "weights")):
            assert torch.equal(got.view(torch.int32), want[key].view(torch.int32)), key
        p_o, n_o, w_o = port.points(ref.disparity, ref.confidence, half.f, half.cx, half.cy, half.baseline)
        assert np.array_equal(pts.cpu().numpy().view(np.uint32), p_o.view(np.uint32))
        assert (p_o[..., 3] > 0).mean() > 0.2
        # without blobs or points: a plain frame
        r2 = s.compute_frame(left, right)
        assert np.array_equal(r2.disparity.view(np.uint32), ref.disparity.view(np.uint32)) and r2.blobs is None


def test_compute_frame_errors(cuda):
    import torch
    from open_source_einstar_b200 import CudaStereo, Errc, RemapTable, SgmParams, StereoError, StereoParams, synth
    pr = synth.raw_objects_pair(seed=2, width=320, height=256, f=275.0, num_disparities=32, n_objects=4, device="cuda")
    (lx, ly), (rx, ry) = pr.maps
    with CudaStereo.create(StereoParams(sgm=SgmParams(min_disparity=pr.min_disparity, num_disparities=32)), 320, 256) as s:
        with pytest.raises(StereoError):
            s.compute_frame(pr.left, pr.right)  # no rectification
        s.set_rectification(RemapTable(lx, ly), RemapTable(rx, ry), 320, 256)
        pts = torch.zeros((256, 320, 4), dtype=torch.float32, device=cuda)
        with pytest.raises(StereoError) as e:  # points without set_point_params
            s.compute_frame(pr.left, pr.right, pts, pts.clone(), torch.zeros((256, 320), device=cuda))
        assert e.value.code == Errc.invalid_argument
        with pytest.raises(StereoError) as e:  # blobs without set_blob_params
            s.compute_frame(pr.left, pr.right, blobs=True)
        assert e.value.code == Errc.invalid_argument


def test_compute_frame_raw_equals_compute_frame(cuda):
    """ds_compute_frame_raw (MetalStereo::compute_frame_raw): the same points, normals and weights as
    compute_frame, the rectified pair as compute_raw returns it, and the reference's errors."""
    import torch
    from open_source_einstar_b200 import (CudaStereo, Errc, RectifiedGeometry, RemapTable, SgmParams, StereoError,
                                          StereoParams, synth)
    pr = synth.raw_objects_pair(seed=12, width=640, height=512, f=560.0, num_disparities=64, n_objects=8, device="cuda")
    (lx, ly), (rx, ry) = pr.maps
    w, h = 320, 256
    sp = StereoParams(sgm=SgmParams(min_disparity=pr.min_disparity // 4 - 2, num_disparities=40), pyramid_levels=1,
                      median=False, detail_enabled=True, filter_occlusion=True, filter_spikes=True,
                      speckle_max_region_size=100)
    geom = RectifiedGeometry(pr.f / 2, (w - 1) / 2.0, (h - 1) / 2.0, pr.baseline, 0.0)
    bufs = lambda: (torch.zeros((h, w, 4), dtype=torch.float32, device=cuda),
                    torch.zeros((h, w, 4), dtype=torch.float32, device=cuda), torch.zeros((h, w), dtype=torch.float32, device=cuda))
    with CudaStereo.create(sp, w, h) as s:
        s.set_rectification(RemapTable(lx, ly), RemapTable(rx, ry), 640, 512)
        p0, n0, w0 = bufs()
        with pytest.raises(StereoError) as e:  # metal_stereo.cpp:254
            s.compute_frame_raw(pr.left, pr.right, p0, n0, w0)
        assert e.value.code == Errc.invalid_argument and "set_point_params" in e.value.message
        s.set_point_params(geom, 150.0, 700.0, 4.0)
        want = s.compute_frame(pr.left, pr.right, p0, n0, w0, rectified=True)
        p1, n1, w1 = bufs()
        rl, rr = s.compute_frame_raw(pr.left, pr.right, p1, n1, w1, rectified=True)
        torch.cuda.synchronize()
        assert np.array_equal(rl, want.rect_left) and np.array_equal(rr, want.rect_right)
        for a, b in ((p0, p1), (n0, n1), (w0, w1)):
            assert torch.equal(a.view(torch.int32), b.view(torch.int32))
        assert s.compute_frame_raw(pr.left, pr.right, p1, n1, w1) is None
